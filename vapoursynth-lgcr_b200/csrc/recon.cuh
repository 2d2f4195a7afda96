// Device-side data layout and helpers of the Recon path.
//
// One FrameJob describes one frame: geometry, parameters, resident tables
// and workspace planes, all in HBM. Every stage kernel takes an array of
// FrameJobs plus a per-stage tile prefix table, so a single launch covers
// one frame (the per-frame form) or a whole batch of uneven frames (the
// batched form); a block finds its frame by binary search over the prefix.
//
// Arithmetic in these kernels follows the reference's scalar build operation
// by operation (the library is compiled with -fmad=false, so no product is
// fused into an add unless written as an fma whose result is provably the
// same). The device helpers restate:
//   bilinear / bilinearFast          src/lgcr.h:467-508
//   principalTensorDirection         src/lgcr.h:516-538
//   lutLookup                        src/lgcr.h:636-641
//   floatToPlane quantizer           src/lgcr.h:997-1013
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lgcr_b200 {

enum SampleKind : int { kU8 = 0, kU16 = 1, kF32 = 2 };

struct AxisView {
    int n, sup;
    const int *start;
    const float *w;          // n * sup
    const double *wd;        // n * sup, the same weights in FP64
    const uint8_t *am;       // n * sup
    const float *wsum, *wabs;
    const float *pos, *lpos;
    const int *cbI0, *lbI0;
    const float *cbF, *lbF;
    const float *kmx, *kss;  // rescue kappa factors per index (separable kernels)
    const uint32_t *amBits;  // per index: bit i set when tap i is active (sup <= 32), or null
};

struct RadialView {
    int valid;
    int supX, supY, phasesX;
    const uint16_t *xPhase, *yPhase;
    const float *weights;
    const float *kappa;      // per phase pair: the guided rescue's kappa, or null
};

// One temporal neighbour of a TRecon frame (TemporalNbr, src/lgcr.h:729-736):
// its chroma and footprint luma map on the chroma grid, and the 16x16 block
// motion field with its confidence, all in HBM.
struct TemporalView {
    const float *U, *V, *lc;           // cw x ch
    const short *mvx, *mvy;            // bw x bh, luma pixels
    const float *conf;                 // bw x bh
    int bw, bh;
};

struct WeightView {          // polyphase resampler table (luma resize etc.)
    int n, sup;
    const int *start;
    const float *w;
};

// Counters written by the sparse stages (per frame).
enum Counter : int {
    kCntActiveOutput = 0,
    kCntActiveChroma = 1,
    kCntSeed = 2,
    kCntMaskPixels = 3,
    kCntRoi = 4,
    kCntCount = 8
};

struct __align__(16) FrameJob {
    // geometry
    int sw, sh, cw, ch, W, H;
    double rw, rh;
    float rwF, rhF;
    int sameSize;
    // input / output
    int inKind, outKind, bits;
    double yScale, cOffset;            // planeToFloat (chroma offset)
    float qScale, qOffC;               // floatToPlane scale / chroma offset
    int maxCode;
    const void *in[3];
    long long inPitch[3];              // bytes
    void *out[3];
    long long outPitch[3];             // bytes
    int writeLuma;                     // copy / resample luma into out[0]
    // parameters
    int algo, kernel, radial, sparse, ridge, cedge, bm;
    int guided;                        // strength > 0
    int useMs, clampHull, trustOn, dil;
    int directOutput;                  // recon kernel quantizes and stores
    int finalInTransfer;               // algo 6: plain (inactive) and detail transfer
                                       // (active pixels) quantize and store
    int needBackProject;
    float strength, sigma, sratio, sdb, stretch, invGsigma2, rescue;
    float strength4;                   // algo 4 selector strength (lambda)
    double support;                    // kernel support (luma radial resize)
    float msStrength, qgate, margin, spOut, trustThr;
    float bpGain;
    float invWxC, invWyC;              // radial AA factors (chroma units)
    float lutScale;
    int lutN;
    const float *lut;
    // tables
    AxisView ax, ay;
    RadialView rad;
    WeightView lumaH, lumaV;           // luma resize (separable)
    const int *lcXb, *lcXe, *lcYb, *lcYe;
    // workspace (packed planes, pitch == width)
    const float *Y, *U, *V;            // source planes as float
    float *Yw, *Uw, *Vw;               // conversion targets (== Y/U/V when converted)
    float *jxx, *jxy, *jyy;            // sw x sh
    float *lc, *ms;                    // cw x ch
    uint8_t *seed;                     // sw x sh trust seed (0/1 bytes)
    uint32_t *mtmp, *mask;             // sw x sh bits: maskWords words per row
    int maskWords;                     // (sw + 31) / 32
    uint8_t *cmask;                    // cw x ch
    float *oU, *oV;                    // W x H float output planes
    float *lumaTmp;                    // W x sh luma resize intermediate
    unsigned long long *counters;      // kCntCount
    float *hTab;                       // W x ch x 8: horizontal sums + window extrema
    float4 *wHull;                     // W x H guided window chroma hull (mnU mxU mnV mxV)
    float2 *wLum;                      // W x H guided window luma extrema (mnL mxL)
    double *uvd;                       // cw x ch x 2: (u, v) in FP64
    uint32_t *actList;                 // active output pixels (y << 16 | x)
    int listed;                        // frame uses the guided work list
    int listGroup;                     // work-list order: output rows per group (1: raster)
    int xferListed;                    // algo 6: detail transfer walks the work list
    uint32_t *chromaList;              // algo 6 sparse: active chroma samples (y << 16 | x)
    int bumpRcpSafe;                   // every guided bump denominator stays below 2^64
    int plainFused;                    // k_plain computes its horizontal rows itself
    int plainRows;                     // output rows per k_plain block
    int noClampX, noClampY;            // every chroma tap index is in range
    // algo 6 / algo 4 / bm workspaces
    float *aff;                        // cw x ch: float4 (aU aV g rng), float4 (mnU mxU
                                       // mnV mxV) per sample, then the dgl plane at 8*C
    float *yc1, *yc2;                  // bilinear / bicubic degradation candidates
    float *ycTmp;                      // cw x sh candidate intermediate (resize case)
    float *detail;                     // sw x sh (or W x H) detail map
    float *detailTmp, *detailTmp2;     // sw x sh scratch
    float *dTab;                       // sw x ch x 4: degraded-luma horizontal pass
    WeightView ycH1, ycV1, ycH2, ycV2; // candidate degradation tables
    WeightView detH, detV;             // detail resample to output (resize)
    int nyqX, nyqY;                    // dyadic Nyquist passes per axis
    int detailFused;                   // k_detail_map builds the detail map in one pass
    int detailRows;                    // output rows per k_detail_map block
    int detailReach;                   // > 0: detail samples farther than this from every
                                       // active pixel are never read (tiles skipped)
    int ycTiled;                       // k_yc_tiled builds the degradation candidates
    int sNoClampX, sNoClampY;          // source-grid axes: every chroma tap index in range
    AxisView sax, say;                 // source-grid plain axes (detail map)
    RadialView srad;
    const float *detailSrc;            // Nyquist-filtered detail on the source grid
    double epsSig;                     // (0.25 sigma)^2
    float sinvWxC, sinvWyC;            // radial AA factors of the source-grid axes
    const int *lsX, *lsY;              // point-sampled luma axes (algo 4)
    const float *lsXf, *lsYf;
    int lgfRoiOnly;
    int blendStores;                   // the selector blend stores the typed output
    int bpStores;                      // back-projection stores the typed output
    float *lgf;                        // 6 chroma planes: aU bU confU aV bV confV
    float *selW2, *selW3;              // W x H routing weights (float algo 4)
    float *gU, *gV;                    // W x H guided values (float algo 4)
    uint8_t *roi;                      // cw x ch
    double lgfEps;
    float *bmAcc;                      // 3 planes W x H (sumU, sumV, weight)
    float *bmGuide;                    // W x H (resized guide when needed)
    int *bmGroups;                     // per anchor: count + match coords
    float *bmPatch;                    // per anchor filtered patches
    int bmAnchorsX, bmAnchorsY;
    const int *bmStartsX, *bmStartsY;
    float bmSigma;
    // TRecon temporal taps (src/recon.cpp:642-745); tnbCount is 0 for Recon
    const TemporalView *tnb;
    int tnbCount;
    int lumaNormalize;                 // float luma copy written as s * 1.0 + 0.0
    int gateDense;                     // mutual gate on every chroma sample (TRecon)
    double shiftXd, shiftYd;           // chroma siting, luma units
    const float *tnwX, *tnwY;          // |sin(pi * frac(mv / r))| per axis, index mv + 64
};

// ---------------------------------------------------------------------------
// scalar helpers with the reference's std:: semantics
// ---------------------------------------------------------------------------
template <class T> __device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }
template <class T> __device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }
template <class T> __device__ __forceinline__ T sclamp(T v, T lo, T hi) {
    return (v < lo) ? lo : (hi < v) ? hi : v;
}
__device__ __forceinline__ int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Running minimum / maximum of an accumulator that starts at +-1e30 (never
// NaN). Float: the hardware min/max (one instruction) returns what the
// reference's std::min/std::max return -- a NaN sample leaves the
// accumulator unchanged either way -- except possibly the sign of a zero
// result, which no output can show (every use is a clamp bound or |x - L0|,
// and the output stores normalise -0 as the reference's s * 1.0 + 0.0 does).
// Double: the std::min/std::max select itself (cheaper here than the
// library fmin/fmax).
__device__ __forceinline__ float runMin(float acc, float v) { return fminf(acc, v); }
__device__ __forceinline__ float runMax(float acc, float v) { return fmaxf(acc, v); }
__device__ __forceinline__ double runMin(double acc, double v) { return (v < acc) ? v : acc; }
__device__ __forceinline__ double runMax(double acc, double v) { return (acc < v) ? v : acc; }

__device__ __forceinline__ float ldf(const float *p) { return __ldg(p); }

// 1/x for denominators of the form 1 + (non-negative terms), i.e. x >= 1,
// equal bit for bit to the IEEE quotient 1.0f / x. On [1, 2^64) the hardware
// approximation (rcp.approx) is refined by one Newton-Raphson step evaluated
// with fused multiply-adds, e = 1 - x*y, y' = y + y*e (Markstein, IBM J. Res.
// Dev. 34(1), 1990); an exhaustive device check over every float in that
// range (lgcr_selftest_reciprocal) finds no difference from 1.0f / x. Larger,
// infinite or NaN arguments take the IEEE division.
constexpr float kRcpFastLimit = 18446744073709551616.0f;   // 2^64

// The IEEE quotient for the rare arguments outside the fast range, kept out
// of line so the unrolled tap loops that call rcpAtLeastOne stay compact.
static __device__ __noinline__ float rcpOutOfRange(float x) { return 1.0f / x; }

// The refinement alone, for callers that have shown x < 2^64 (or NaN, which
// it returns as the division would).
__device__ __forceinline__ float rcpInRange(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    const float e = __fmaf_rn(-x, y, 1.0f);
    return __fmaf_rn(y, e, y);
}

__device__ __forceinline__ float rcpAtLeastOne(float x) {
    if (x < kRcpFastLimit)
        return rcpInRange(x);
    return rcpOutOfRange(x);
}

// Two lanes of FP32 arithmetic per instruction: the packed f32x2 add, sub,
// mul and fma of sm_100 round each lane exactly like the scalar instruction.
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pk2(float a, float b) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void up2(f32x2 r, float &a, float &b) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
// Dilated trust mask bit of luma sample (x, y).
__device__ __forceinline__ uint32_t maskAt(const FrameJob &J, int x, int y) {
    return (__ldg(J.mask + (size_t)y * J.maskWords + (x >> 5)) >> (x & 31)) & 1u;
}

// Shared-memory copy of one frame's job for the whole block. Kernels that
// read FrameJob fields inside loops with global stores read them from this
// copy, so the fields are not reloaded from global memory after each store.
__device__ __forceinline__ void stageJob(const FrameJob *__restrict__ jobs, int f, FrameJob &s) {
    const int4 *src = reinterpret_cast<const int4 *>(jobs + f);
    int4 *dst = reinterpret_cast<int4 *>(&s);
    const int tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    for (int i = tid; i < (int)(sizeof(FrameJob) / 16); i += nthreads)
        dst[i] = __ldg(src + i);
    __syncthreads();
}

// Block -> frame by binary search over the stage prefix table.
__device__ __forceinline__ int findFrame(const int *tileStart, int njobs, int block) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(tileStart + mid) <= block) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// lgcr.h:467-475: bilinear sample with clamped fetches at a (double) position
// that is always a float value here; the fraction is exact in float.
__device__ __forceinline__ float bilinearAt(const float *p, int w, int h, float xf, float yf) {
    const float flx = floorf(xf), fly = floorf(yf);
    const int x0 = (int)flx, y0 = (int)fly;
    const float fx = xf - flx;
    const float fy = yf - fly;
    const int xa = iclamp(x0, 0, w - 1), xb = iclamp(x0 + 1, 0, w - 1);
    const int ya = iclamp(y0, 0, h - 1), yb = iclamp(y0 + 1, 0, h - 1);
    const float a = ldf(p + (size_t)ya * w + xa), b = ldf(p + (size_t)ya * w + xb);
    const float c = ldf(p + (size_t)yb * w + xa), d = ldf(p + (size_t)yb * w + xb);
    return a + (b - a) * fx + (c - a) * fy + (a - b - c + d) * fx * fy;
}

// lgcr.h:494-508: 4 direct loads with pre-clamped axis indices. Planes are
// packed, so reads index the flat array exactly as the reference does.
__device__ __forceinline__ float bilinearFast(const float *p, int w, int h, int x0, float fx,
                                              int y0, float fy) {
    if (w == 1) {
        const float a = ldf(p + (size_t)y0 * w);
        if (h == 1)
            return a;
        const float c = ldf(p + (size_t)(y0 + 1) * w);
        return a + (c - a) * fy;
    }
    const float *r0 = p + (size_t)y0 * w + x0;
    if (h == 1)
        return ldf(r0) + (ldf(r0 + 1) - ldf(r0)) * fx;
    const float *r1 = r0 + w;
    const float a = ldf(r0), b = ldf(r0 + 1), c = ldf(r1), d = ldf(r1 + 1);
    return a + (b - a) * fx + (c - a) * fy + (a - b - c + d) * fx * fy;
}

// bilinearFast of four interleaved planes (float4 per sample): the same
// loads' positions and the same arithmetic per component.
__device__ __forceinline__ float4 bl4(float4 a, float4 b, float4 c, float4 d, float fx, float fy) {
    return make_float4(a.x + (b.x - a.x) * fx + (c.x - a.x) * fy + (a.x - b.x - c.x + d.x) * fx * fy,
                       a.y + (b.y - a.y) * fx + (c.y - a.y) * fy + (a.y - b.y - c.y + d.y) * fx * fy,
                       a.z + (b.z - a.z) * fx + (c.z - a.z) * fy + (a.z - b.z - c.z + d.z) * fx * fy,
                       a.w + (b.w - a.w) * fx + (c.w - a.w) * fy + (a.w - b.w - c.w + d.w) * fx * fy);
}

__device__ __forceinline__ float4 bilinearFast4(const float4 *p, int w, int h, int x0, float fx,
                                                int y0, float fy) {
    if (w == 1) {
        const float4 a = __ldg(p + (size_t)y0 * w);
        if (h == 1)
            return a;
        const float4 c = __ldg(p + (size_t)(y0 + 1) * w);
        return make_float4(a.x + (c.x - a.x) * fy, a.y + (c.y - a.y) * fy, a.z + (c.z - a.z) * fy,
                           a.w + (c.w - a.w) * fy);
    }
    const float4 *r0 = p + (size_t)y0 * w + x0;
    if (h == 1) {
        const float4 a = __ldg(r0), b = __ldg(r0 + 1);
        return make_float4(a.x + (b.x - a.x) * fx, a.y + (b.y - a.y) * fx, a.z + (b.z - a.z) * fx,
                           a.w + (b.w - a.w) * fx);
    }
    const float4 *r1 = r0 + w;
    return bl4(__ldg(r0), __ldg(r0 + 1), __ldg(r1), __ldg(r1 + 1), fx, fy);
}

struct TensorDir { float coherence, nx, ny; };

// lgcr.h:516-538
__device__ __forceinline__ TensorDir principalDirection(float jxx, float jxy, float jyy) {
    TensorDir d{0.0f, 1.0f, 0.0f};
    const float difference = jxx - jyy;
    const float sum = jxx + jyy;
    const float cross = 2.0f * jxy;
    const float disc = sqrtf(difference * difference + cross * cross);
    d.coherence = disc / (sum + 1e-12f);
    if (disc <= 1e-20f)
        return d;
    float vx, vy;
    if (difference >= 0.0f) {
        vx = disc + difference;
        vy = cross;
    } else {
        vx = cross;
        vy = disc - difference;
    }
    const float inv = 1.0f / sqrtf(vx * vx + vy * vy);
    d.nx = vx * inv;
    d.ny = vy * inv;
    return d;
}

// lgcr.h:636-641
__device__ __forceinline__ float lutLookupDev(const float *lut, int n, float idx) {
    int i0 = (int)idx;
    i0 = iclamp(i0, 0, n - 2);
    const float fr = smin(idx - (float)i0, 1.0f);
    const float a = ldf(lut + i0);
    return a + (ldf(lut + i0 + 1) - a) * fr;
}

// lgcr.h:1008: int(s*scale + off + 0.5f), clamped.
__device__ __forceinline__ int quantize(float s, float scale, float off, int maxCode) {
    const float t = s * scale + off + 0.5f;
    const int v = __float2int_rz(t);
    return v < 0 ? 0 : (v > maxCode ? maxCode : v);
}

// Store one chroma output sample in the output plane's type.
__device__ __forceinline__ void storeChroma(const FrameJob &J, int plane, int x, int y, float v) {
    char *row = static_cast<char *>(J.out[plane]) + (long long)y * J.outPitch[plane];
    if (J.outKind == kF32) {
        reinterpret_cast<float *>(row)[x] = v + 0.0f;   // s*1.0+0.0 in the reference
    } else {
        const int q = quantize(v, J.qScale, J.qOffC, J.maxCode);
        if (J.outKind == kU8) reinterpret_cast<uint8_t *>(row)[x] = (uint8_t)q;
        else reinterpret_cast<uint16_t *>(row)[x] = (uint16_t)q;
    }
}

__device__ __forceinline__ void storeLuma(const FrameJob &J, int x, int y, float v) {
    char *row = static_cast<char *>(J.out[0]) + (long long)y * J.outPitch[0];
    if (J.outKind == kF32) {
        reinterpret_cast<float *>(row)[x] = v + 0.0f;
    } else {
        const int q = quantize(v, J.qScale, 0.0f, J.maxCode);
        if (J.outKind == kU8) reinterpret_cast<uint8_t *>(row)[x] = (uint8_t)q;
        else reinterpret_cast<uint16_t *>(row)[x] = (uint16_t)q;
    }
}

// Jinc selector frames whose guided pass also forms the radial plain base of
// its listed pixels (pass 1 of the guided pixel): the plain stage skips
// those pixels and the batch launches the guided kernel instance that has
// the fused pass (the host decides with this same test).
__host__ __device__ __forceinline__ bool radialPlainFused(const FrameJob &J) {
    return J.guided && J.radial && J.algo == 4 && J.rad.valid && J.rad.supX == J.ax.sup &&
           J.rad.supY == J.ay.sup && J.noClampX && J.noClampY && J.ax.sup == J.ay.sup &&
           (J.ax.sup == 4 || J.ax.sup == 6 || J.ax.sup == 8);
}

} // namespace lgcr_b200
