// Map-building stages of the Recon path (all HBM-bound stencils):
//   k_convert      planeToFloat                  src/lgcr.h:986-995
//                  + buildLcMap footprint sums    src/maps.cpp:425-499
//   k_tensor       sobelTensor3x3 + trust seed   src/maps.cpp:9-168
//   k_dilate_h/v   buildTrustMask dilation       src/maps.cpp:280-340
//   k_mark_chroma  buildSparseWorkset            src/maps.cpp:342-422
//   k_count        active chroma samples         src/maps.cpp:398-420
//   k_gate         buildMutualGate               src/maps.cpp:831-948
//
// The dilated trust mask is stored one bit per luma sample (rows of
// maskWords 32-bit words, bit i of word k = column 32k + i): the dilation
// runs on whole words and later stages test single bits.
#include "kernels.cuh"

namespace lgcr_b200 {

// ---------------------------------------------------------------------------
// Input conversion with the footprint luma map folded in. A warp converts
// one row segment (kConvertLumaSpan luma samples, 8 consecutive per lane and
// both halves' loads in flight together; kConvertSpan chroma samples, lane l
// taking samples l, l + 32, ...), so every load and store is coalesced. The
// first convertLumaBlocks(J) blocks of a frame cover the luma plane (and copy
// it to a same-size output), the rest the chroma planes; the chroma blocks
// also clear the chroma work masks and compute lc from the luma codes.
// ---------------------------------------------------------------------------
// Sample access specialised on the sample type (row pointers hoisted).
template <int KIND>
__device__ __forceinline__ uint32_t rawLoad(const char *row, int x) {
    if (KIND == kU16)
        return __ldg(reinterpret_cast<const unsigned short *>(row) + x);
    if (KIND == kU8)
        return __ldg(reinterpret_cast<const unsigned char *>(row) + x);
    return __float_as_uint(__ldg(reinterpret_cast<const float *>(row) + x));
}

template <int KIND>
__device__ __forceinline__ void rawStore(char *row, int x, uint32_t raw) {
    if (KIND == kU16) reinterpret_cast<unsigned short *>(row)[x] = (unsigned short)raw;
    else if (KIND == kU8) reinterpret_cast<unsigned char *>(row)[x] = (unsigned char)raw;
    else reinterpret_cast<uint32_t *>(row)[x] = raw;
}

// planeToFloat of one sample: s * scale + offset in double, then float.
template <int KIND>
__device__ __forceinline__ float rawToFloat(uint32_t raw, double scale, double off) {
    return KIND == kF32 ? __uint_as_float(raw) : (float)((double)raw * scale + off);
}

// Eight consecutive raw samples from one 16-byte (u16, f32: two) or 8-byte
// (u8) aligned load; false when the address is not aligned.
template <int KIND>
__device__ __forceinline__ bool rawLoad8(const char *row, int x, uint32_t (&raw)[8]) {
    constexpr int bps = KIND == kF32 ? 4 : (KIND == kU16 ? 2 : 1);
    const char *p = row + (size_t)x * bps;
    if (KIND == kU8) {
        if (reinterpret_cast<uintptr_t>(p) & 7)
            return false;
        const uint2 q = __ldg(reinterpret_cast<const uint2 *>(p));
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            raw[k] = (q.x >> (8 * k)) & 0xffu;
            raw[4 + k] = (q.y >> (8 * k)) & 0xffu;
        }
        return true;
    }
    if (reinterpret_cast<uintptr_t>(p) & 15)
        return false;
    if (KIND == kU16) {
        const uint4 q = __ldg(reinterpret_cast<const uint4 *>(p));
        const uint32_t w[4] = { q.x, q.y, q.z, q.w };
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            raw[2 * k] = w[k] & 0xffffu;
            raw[2 * k + 1] = w[k] >> 16;
        }
        return true;
    }
    const uint4 a = __ldg(reinterpret_cast<const uint4 *>(p)), b = __ldg(reinterpret_cast<const uint4 *>(p) + 1);
    raw[0] = a.x; raw[1] = a.y; raw[2] = a.z; raw[3] = a.w;
    raw[4] = b.x; raw[5] = b.y; raw[6] = b.z; raw[7] = b.w;
    return true;
}

template <int KIND>
__device__ __forceinline__ void rawStore8(char *row, int x, const uint32_t (&raw)[8]) {
    constexpr int bps = KIND == kF32 ? 4 : (KIND == kU16 ? 2 : 1);
    char *p = row + (size_t)x * bps;
    if (KIND == kU16 && !(reinterpret_cast<uintptr_t>(p) & 15)) {
        *reinterpret_cast<uint4 *>(p) = make_uint4(raw[0] | raw[1] << 16, raw[2] | raw[3] << 16,
                                                   raw[4] | raw[5] << 16, raw[6] | raw[7] << 16);
        return;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k)
        rawStore<KIND>(row, x + k, raw[k]);
}

// floatToPlane of a float sample (s * 1.0 + 0.0): the same bits except that
// a negative zero becomes +0.
__device__ __forceinline__ uint32_t normalizedFloat(uint32_t raw) {
    return __float_as_uint(__uint_as_float(raw) + 0.0f);
}

// Luma: each lane converts 8 consecutive samples (one vector load) in each
// half of the warp's row segment, both loads issued before any store;
// unaligned rows take the per-sample path.
template <int KIND>
__device__ __forceinline__ void convertLuma(const FrameJob &J, int y, int xb, int lane) {
    const char *src = static_cast<const char *>(J.in[0]) + (long long)y * J.inPitch[0];
    char *dst = (J.writeLuma && J.sameSize) ? static_cast<char *>(J.out[0]) + (long long)y * J.outPitch[0]
                                            : nullptr;
    float *yw = J.Yw ? J.Yw + (size_t)y * J.sw : nullptr;
    const double scale = J.yScale;
    const int w = J.sw;
    constexpr int half = kConvertLumaSpan / 2;
    uint32_t raw[2][8];
    bool vec[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int x = xb + s * half + lane * 8;
        vec[s] = x + 8 <= w && rawLoad8<KIND>(src, x, raw[s]);
    }
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int x = xb + s * half + lane * 8;
        if (x >= w)
            continue;
        if (vec[s]) {
            if (yw) {
                float v[8];
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    v[k] = rawToFloat<KIND>(raw[s][k], scale, 0.0);
                if (!(reinterpret_cast<uintptr_t>(yw + x) & 15)) {
                    reinterpret_cast<float4 *>(yw + x)[0] = make_float4(v[0], v[1], v[2], v[3]);
                    reinterpret_cast<float4 *>(yw + x)[1] = make_float4(v[4], v[5], v[6], v[7]);
                } else {
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        yw[x + k] = v[k];
                }
            }
            if (dst) {
                if (KIND == kF32 && J.lumaNormalize) {
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        raw[s][k] = normalizedFloat(raw[s][k]);
                }
                rawStore8<KIND>(dst, x, raw[s]);
            }
            continue;
        }
        for (int k = 0; k < 8 && x + k < w; ++k) {
            const uint32_t r = rawLoad<KIND>(src, x + k);
            if (yw)
                yw[x + k] = rawToFloat<KIND>(r, scale, 0.0);
            if (dst)
                rawStore<KIND>(dst, x + k, (KIND == kF32 && J.lumaNormalize) ? normalizedFloat(r) : r);
        }
    }
}

// Chroma: groups of two samples per lane; a group's loads (U, V and, for
// the usual 2x2 footprint, the four luma codes of lc) are issued before its
// stores, which go through restrict-qualified pointers.
template <int KIND>
__device__ __forceinline__ void convertChroma(const FrameJob &J, int cy, int xb, int lane) {
    const char *su = static_cast<const char *>(J.in[1]) + (long long)cy * J.inPitch[1];
    const char *sv = static_cast<const char *>(J.in[2]) + (long long)cy * J.inPitch[2];
    const size_t rowOff = (size_t)cy * J.cw;
    const double scale = J.yScale, off = J.cOffset;
    float *__restrict__ uw = J.Uw;
    float *__restrict__ vw = J.Vw;
    double2 *__restrict__ uvd = reinterpret_cast<double2 *>(J.uvd);
    uint8_t *__restrict__ cmask = J.cmask;
    uint8_t *__restrict__ roi = J.roi;
    float *__restrict__ lc = J.lc;
    int yb = 0, ye = 0;
    const char *lrow0 = nullptr;
    const long long lpitch = J.inPitch[0];
    if (lc) {
        yb = __ldg(J.lcYb + cy);
        ye = __ldg(J.lcYe + cy);
        lrow0 = static_cast<const char *>(J.in[0]) + (long long)yb * lpitch;
    }
    constexpr int kGroup = 2;
#pragma unroll 1
    for (int g = 0; g < kConvertSpan / 32; g += kGroup) {
        uint32_t ru[kGroup], rv[kGroup], fp[kGroup][4];
        int fxb[kGroup], fxe[kGroup];
#pragma unroll
        for (int k = 0; k < kGroup; ++k) {
            const int cx = xb + lane + 32 * (g + k);
            if (cx >= J.cw)
                break;
            ru[k] = rawLoad<KIND>(su, cx);
            rv[k] = rawLoad<KIND>(sv, cx);
            if (lc) {
                fxb[k] = __ldg(J.lcXb + cx);
                fxe[k] = __ldg(J.lcXe + cx);
                if (fxe[k] - fxb[k] == 2 && ye - yb == 2) {
                    fp[k][0] = rawLoad<KIND>(lrow0, fxb[k]);
                    fp[k][1] = rawLoad<KIND>(lrow0, fxb[k] + 1);
                    fp[k][2] = rawLoad<KIND>(lrow0 + lpitch, fxb[k]);
                    fp[k][3] = rawLoad<KIND>(lrow0 + lpitch, fxb[k] + 1);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kGroup; ++k) {
            const int cx = xb + lane + 32 * (g + k);
            if (cx >= J.cw)
                break;
            const size_t o = rowOff + cx;
            const float u = rawToFloat<KIND>(ru[k], scale, off);
            const float v = rawToFloat<KIND>(rv[k], scale, off);
            if (uw) uw[o] = u;
            if (vw) vw[o] = v;
            if (uvd) uvd[o] = make_double2((double)u, (double)v);
            if (cmask) cmask[o] = 0;
            if (roi) roi[o] = 0;
            if (lc) {
                // buildLcMap: raster-order double sum over the footprint
                const int xb0 = fxb[k], xe0 = fxe[k];
                double sum = 0.0;
                if (xe0 - xb0 == 2 && ye - yb == 2) {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        sum += (double)rawToFloat<KIND>(fp[k][q], scale, 0.0);
                } else {
                    const char *lrow = lrow0;
                    for (int j = yb; j < ye; ++j, lrow += lpitch)
                        for (int i = xb0; i < xe0; ++i)
                            sum += (double)rawToFloat<KIND>(rawLoad<KIND>(lrow, i), scale, 0.0);
                }
                lc[o] = (float)(sum / ((double)(xe0 - xb0) * (double)(ye - yb)));
            }
        }
    }
}

__global__ void __launch_bounds__(kConvertWarps * 32, 3)
k_convert(LGCR_STAGE_ARGS) {
    __shared__ FrameJob sJob;
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    stageJob(jobs, f, sJob);
    const FrameJob &J = sJob;
    const int tile = blockIdx.x - tileStart[f];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int lumaBlocks = convertLumaBlocks(J.sw, J.sh);
    if (tile < lumaBlocks) {
        const int gpr = (J.sw + kConvertLumaSpan - 1) / kConvertLumaSpan;
        const int gw = tile * kConvertWarps + warp;
        if (gw >= J.sh * gpr)
            return;
        if (gw == 0 && lane < kCntCount)
            J.counters[lane] = 0ull;
        const int y = gw / gpr, xb = (gw % gpr) * kConvertLumaSpan;
        switch (J.inKind) {
        case kU8: convertLuma<kU8>(J, y, xb, lane); break;
        case kU16: convertLuma<kU16>(J, y, xb, lane); break;
        default: convertLuma<kF32>(J, y, xb, lane); break;
        }
        return;
    }
    const int gpr = (J.cw + kConvertSpan - 1) / kConvertSpan;
    const int gw = (tile - lumaBlocks) * kConvertWarps + warp;
    if (gw >= J.ch * gpr)
        return;
    const int cy = gw / gpr, xb = (gw % gpr) * kConvertSpan;
    switch (J.inKind) {
    case kU8: convertChroma<kU8>(J, cy, xb, lane); break;
    case kU16: convertChroma<kU16>(J, cy, xb, lane); break;
    default: convertChroma<kF32>(J, cy, xb, lane); break;
    }
}

// ---------------------------------------------------------------------------
// Structure tensor: Sobel/8 gradients at clamped positions, vertical 3-row
// sums of the outer products, horizontal 3-tap box with the reference's
// border rule ((2a+b)/9 and (a+2b)/9 at the ends, *(1/9) inside), trust
// seed jxx + jyy > thr.
//
// Each warp walks down a strip of kTensorRows rows over 32 consecutive
// columns x0-2 .. x0+29 and emits the 28 middle ones: lane values are luma
// samples at clamped columns, horizontal neighbours come from shuffles, the
// three gradient rows and their products roll in registers. The warps of a
// block sit side by side.
// ---------------------------------------------------------------------------
struct Tri { float l, m, r; };

__device__ __forceinline__ Tri tri(float v) {
    return { __shfl_up_sync(0xffffffffu, v, 1), v, __shfl_down_sync(0xffffffffu, v, 1) };
}

// t = row above, c = centre row, b = row below (maps.cpp Sobel/8 order)
__device__ __forceinline__ void sobel(const Tri &t, const Tri &c, const Tri &b, float &gx, float &gy) {
    gx = (t.r + 2.0f * c.r + b.r - t.l - 2.0f * c.l - b.l) * 0.125f;
    gy = (b.l + 2.0f * b.m + b.r - t.l - 2.0f * t.m - t.r) * 0.125f;
}

__global__ void __launch_bounds__(kTensorWarps * 32)
k_tensor(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int w = J.sw, h = J.sh;
    constexpr int span = kTensorCols * kTensorWarps;
    const int tilesX = (w + span - 1) / span;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x0 = (tile % tilesX) * span + warp * kTensorCols;
    if (x0 >= w)
        return;                                   // whole warp
    const int y0 = (tile / tilesX) * kTensorRows;
    const int y1 = min(y0 + kTensorRows, h);
    const int c = x0 - 2 + lane;
    const bool emitLane = lane >= 2 && lane < 2 + kTensorCols && c < w;
    const float *col = J.Y + iclamp(c, 0, w - 1);
    auto L = [&](int r) { return ldf(col + (size_t)iclamp(r, 0, h - 1) * w); };

    // G(r) = gradient at row clamp(r); prologue G(y0-1), G(y0)
    const Tri la = tri(L(y0 - 2)), lb = tri(L(y0 - 1));
    Tri rm = tri(L(y0)), rn = tri(L(y0 + 1));
    float gxA, gyA, gxB, gyB;
    sobel(lb, rm, rn, gxB, gyB);
    if (y0 == 0) {
        gxA = gxB;
        gyA = gyB;
    } else {
        sobel(la, lb, rm, gxA, gyA);
    }
    float pxxA = gxA * gxA, pxyA = gxA * gyA, pyyA = gyA * gyA;
    float pxxB = gxB * gxB, pxyB = gxB * gyB, pyyB = gyB * gyB;
    const float ninth = 1.0f / 9.0f;
    const float thr = J.trustThr;
    float pf = L(y0 + 2);
    for (int y = y0; y < y1; ++y) {
        const Tri re = tri(pf);                   // luma row clamp(y + 2)
        pf = L(y + 3);
        float gxC, gyC;
        if (y + 1 < h) {
            sobel(rm, rn, re, gxC, gyC);
        } else {
            gxC = gxB;
            gyC = gyB;
        }
        const float pxxC = gxC * gxC, pxyC = gxC * gyC, pyyC = gyC * gyC;
        const float vxx = pxxA + pxxB + pxxC;
        const float vxy = pxyA + pxyB + pxyC;
        const float vyy = pyyA + pyyB + pyyC;
        const float lxx = __shfl_up_sync(0xffffffffu, vxx, 1), rxx = __shfl_down_sync(0xffffffffu, vxx, 1);
        const float lxy = __shfl_up_sync(0xffffffffu, vxy, 1), rxy = __shfl_down_sync(0xffffffffu, vxy, 1);
        const float lyy = __shfl_up_sync(0xffffffffu, vyy, 1), ryy = __shfl_down_sync(0xffffffffu, vyy, 1);
        if (emitLane) {
            float oxx, oxy, oyy;
            if (c == 0) {
                const bool wide = w > 1;
                oxx = (2.0f * vxx + (wide ? rxx : vxx)) / 9.0f;
                oxy = (2.0f * vxy + (wide ? rxy : vxy)) / 9.0f;
                oyy = (2.0f * vyy + (wide ? ryy : vyy)) / 9.0f;
            } else if (c == w - 1) {
                oxx = (lxx + 2.0f * vxx) / 9.0f;
                oxy = (lxy + 2.0f * vxy) / 9.0f;
                oyy = (lyy + 2.0f * vyy) / 9.0f;
            } else {
                oxx = ninth * (lxx + vxx + rxx);
                oxy = ninth * (lxy + vxy + rxy);
                oyy = ninth * (lyy + vyy + ryy);
            }
            const size_t o = (size_t)y * w + c;
            J.jxx[o] = oxx;
            J.jxy[o] = oxy;
            J.jyy[o] = oyy;
            if (J.trustOn)
                J.seed[o] = (oxx + oyy > thr) ? 1 : 0;
        }
        pxxA = pxxB; pxyA = pxyB; pyyA = pyyB;
        pxxB = pxxC; pxyB = pxyC; pyyB = pyyC;
        gxB = gxC; gyB = gyC;
        rm = rn;
        rn = re;
    }
}

// ---------------------------------------------------------------------------
// Trust-mask dilation: square window of radius r clipped to the plane (the
// reference's rolling population counts give the same set).
// Horizontal: one block per row packs the seed bytes into words in shared
// memory and ORs the word stream shifted by 1..r either way (funnel shifts
// across word boundaries). Needs r <= 32 * (kDilPadWords - 1).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t packNibble(uint32_t fourBytes) {
    // bytes are 0 or 1: the product gathers byte i at bit 21 + i
    return ((fourBytes * 0x204081u) >> 21) & 0xFu;
}

__global__ void __launch_bounds__(128)
k_dilate_h(LGCR_STAGE_ARGS) {
    __shared__ uint32_t words[kDilMaxWords + 2 * kDilPadWords];
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int y = blockIdx.x - tileStart[f];
    const int w = J.sw, mw = J.maskWords, r = J.dil;
    const uint8_t *src = J.seed + (size_t)y * w;
    for (int k = threadIdx.x; k < mw + 2 * kDilPadWords; k += blockDim.x) {
        const int wk = k - kDilPadWords;
        uint32_t bits = 0;
        if (wk >= 0 && wk < mw) {
            const int x = wk * 32;
            const uint8_t *p = src + x;
            if (x + 32 <= w && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
                const uint4 a = __ldg(reinterpret_cast<const uint4 *>(p));
                const uint4 b = __ldg(reinterpret_cast<const uint4 *>(p) + 1);
                bits = packNibble(a.x) | packNibble(a.y) << 4 | packNibble(a.z) << 8 |
                       packNibble(a.w) << 12 | packNibble(b.x) << 16 | packNibble(b.y) << 20 |
                       packNibble(b.z) << 24 | packNibble(b.w) << 28;
            } else {
                const int n = min(32, w - x);
                for (int i = 0; i < n; ++i)
                    bits |= (p[i] != 0 ? 1u : 0u) << i;
            }
        }
        words[k] = bits;
    }
    __syncthreads();
    const int qmax = r >> 5;
    for (int k = threadIdx.x; k < mw; k += blockDim.x) {
        const uint32_t *W = words + kDilPadWords + k;
        uint32_t acc = W[0];
        for (int q = 0; q <= qmax; ++q) {
            const uint32_t r0 = W[q], r1 = W[q + 1], l0 = W[-q], l1 = W[-q - 1];
            if (q > 0)
                acc |= r0 | l0;
            const int smax = min(31, r - 32 * q);
            for (int s = 1; s <= smax; ++s)
                acc |= __funnelshift_r(r0, r1, s) | __funnelshift_l(l1, l0, s);
        }
        if (k == mw - 1 && (w & 31))
            acc &= (1u << (w & 31)) - 1u;
        J.mtmp[(size_t)y * mw + k] = acc;
    }
}

// Vertical: one thread per mask word, OR over rows y-r .. y+r (clipped).
// Also counts the set mask samples (one atomic per block).
__global__ void __launch_bounds__(256)
k_dilate_v(LGCR_STAGE_ARGS) {
    __shared__ unsigned warpSum[8];
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int mw = J.maskWords, h = J.sh, r = J.dil;
    const int tilesX = (mw + 31) / 32;
    const int k = (tile % tilesX) * 32 + threadIdx.x;
    const int y = (tile / tilesX) * 8 + threadIdx.y;
    unsigned count = 0;
    if (k < mw && y < h) {
        const int lo = max(0, y - r), hi = min(h - 1, y + r);
        const uint32_t *col = J.mtmp + k;
        uint32_t acc = 0;
        for (int j = lo; j <= hi; ++j)
            acc |= __ldg(col + (size_t)j * mw);
        J.mask[(size_t)y * mw + k] = acc;
        count = __popc(acc);
    }
    for (int o = 16; o > 0; o >>= 1)
        count += __shfl_down_sync(0xffffffffu, count, o);
    const int tid = threadIdx.y * 32 + threadIdx.x;
    if ((tid & 31) == 0)
        warpSum[tid >> 5] = count;
    __syncthreads();
    if (tid == 0) {
        unsigned total = 0;
        for (int i = 0; i < 8; ++i)
            total += warpSum[i];
        if (total)
            atomicAdd(J.counters + kCntMaskPixels, (unsigned long long)total);
    }
}

// ---------------------------------------------------------------------------
// Sparse workset: a block covers 256 consecutive 32-pixel words of the
// output rows in row-group order (markWord); each warp takes 32 of them in
// turn, one pixel per lane. An output pixel is active when the mask sample
// its position maps to is set (every pixel when the frame is not sparse);
// active pixels mark the 2x2 chroma bilinear footprint. The block counts its
// active pixels, takes one range of the frame's guided work list with one
// atomic, and the lanes append their pixels (y << 16 | x) in word order at
// their prefix offsets.
// ---------------------------------------------------------------------------
// Word idx of the frame's list order: groups of G = J.listGroup output
// rows, a group's words column by column, each column's rows in turn (G = 1:
// raster order).
__device__ __forceinline__ void markWord(int idx, int ow, int G, int &oy, int &kw) {
    G = G < 1 ? 1 : G;
    const int per = ow * G;
    const int g = idx / per, rem = idx - g * per;
    kw = rem / G;
    oy = g * G + (rem - kw * G);
}

__device__ __forceinline__ uint32_t activeWord(const FrameJob &J, int kw, int oy) {
    const int x0 = kw * 32;
    const int n = min(32, J.W - x0);
    const uint32_t valid = n == 32 ? 0xffffffffu : ((1u << n) - 1u);
    if (!J.sparse)
        return valid;
    if (J.sameSize)
        return __ldg(J.mask + (size_t)oy * J.maskWords + kw) & valid;
    const int my = min(J.sh - 1, (int)((long long)oy * J.sh / J.H));
    uint32_t bits = 0;
    for (int i = 0; i < n; ++i) {
        const int mx = min(J.sw - 1, (int)((long long)(x0 + i) * J.sw / J.W));
        bits |= maskAt(J, mx, my) << i;
    }
    return bits;
}

__global__ void __launch_bounds__(256)
k_mark_chroma(LGCR_STAGE_ARGS) {
    __shared__ unsigned warpCount[8];
    __shared__ unsigned long long blockBase;
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int ow = (J.W + 31) / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wordBase = tile * 256 + warp * 32;          // this warp's 32 words
    // pass 1: lane i counts word wordBase + i (and keeps its position for
    // pass 2, where the warp walks the words by shuffles)
    uint32_t myBits = 0;
    int myOy, myKw;
    markWord(wordBase + lane, ow, J.listGroup, myOy, myKw);
    if (myOy < J.H)
        myBits = activeWord(J, myKw, myOy);
    const unsigned cnt = __popc(myBits);
    unsigned incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned n = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += n;
    }
    if (lane == 31)
        warpCount[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned total = 0;
        for (int i = 0; i < 8; ++i) {
            const unsigned c = warpCount[i];
            warpCount[i] = total;
            total += c;
        }
        blockBase = total ? atomicAdd(J.counters + kCntActiveOutput, (unsigned long long)total) : 0ull;
    }
    __syncthreads();
    const unsigned long long warpBase = blockBase + warpCount[warp];
    const unsigned excl = incl - cnt;
    const uint32_t below = (1u << lane) - 1u;
    // pass 2: the warp walks its words, one pixel per lane
    for (int i = 0; i < 32; ++i) {
        const uint32_t bits = __shfl_sync(0xffffffffu, myBits, i);
        const unsigned offs = __shfl_sync(0xffffffffu, excl, i);
        if (!bits)
            continue;                                      // warp-uniform
        const int oy = __shfl_sync(0xffffffffu, myOy, i);
        const int kw = __shfl_sync(0xffffffffu, myKw, i);
        if (!((bits >> lane) & 1u))
            continue;
        const int ox = kw * 32 + lane;
        if (J.sparse) {
            const int cy0 = __ldg(J.ay.cbI0 + oy);
            const int cy1 = min(cy0 + 1, J.ch - 1);
            const int cx0 = __ldg(J.ax.cbI0 + ox);
            const int cx1 = min(cx0 + 1, J.cw - 1);
            uint8_t *row0 = J.cmask + (size_t)cy0 * J.cw;
            uint8_t *row1 = J.cmask + (size_t)cy1 * J.cw;
            row0[cx0] = 1; row0[cx1] = 1;
            row1[cx0] = 1; row1[cx1] = 1;
        }
        if (J.listed || J.xferListed)
            J.actList[warpBase + offs + __popc(bits & below)] = ((uint32_t)oy << 16) | (uint32_t)ox;
    }
}

// Active chroma samples: population count of the 0/1 chroma mask bytes, a
// contiguous 64-byte span per thread, one atomic per block. Frames with a
// chroma work list also get their active samples (y << 16 | x) appended in
// raster order at the block's range.
__global__ void __launch_bounds__(256)
k_count(LGCR_STAGE_ARGS) {
    __shared__ unsigned warpSum[8];
    __shared__ unsigned long long blockBase;
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const size_t nc = (size_t)J.cw * J.ch;
    const size_t span = (size_t)tile * kCountChunk + (size_t)threadIdx.x * (kCountChunk / 256);
    const size_t spanEnd = min(nc, span + kCountChunk / 256);
    unsigned c = 0;
    if (span + kCountChunk / 256 <= nc) {
#pragma unroll
        for (int k = 0; k < kCountChunk / 256 / 16; ++k) {
            const uint4 q = __ldg(reinterpret_cast<const uint4 *>(J.cmask + span) + k);
            c += __popc(q.x) + __popc(q.y) + __popc(q.z) + __popc(q.w);
        }
    } else {
        for (size_t k = span; k < spanEnd; ++k)
            c += J.cmask[k] != 0;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned incl = c;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned n = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += n;
    }
    if (lane == 31)
        warpSum[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned total = 0;
        for (int i = 0; i < 8; ++i) {
            const unsigned w = warpSum[i];
            warpSum[i] = total;
            total += w;
        }
        blockBase = total ? atomicAdd(J.counters + kCntActiveChroma, (unsigned long long)total) : 0ull;
    }
    __syncthreads();
    if (J.chromaList && c) {
        unsigned long long pos = blockBase + warpSum[warp] + incl - c;
        int y = (int)(span / (size_t)J.cw);
        int x = (int)(span - (size_t)y * J.cw);
        for (size_t k = span; k < spanEnd; ++k) {
            if (J.cmask[k])
                J.chromaList[pos++] = ((uint32_t)y << 16) | (uint32_t)x;
            if (++x == J.cw) {
                x = 0;
                ++y;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Mutual-structure gate at chroma resolution. Gradients of lc, U, V are
// computed in shared memory for the tile plus a 4-pixel halo (the farthest
// any gate sample reaches), at clamped positions, exactly as the reference's
// dense Sobel rows; the sparse reference computes the same values wherever
// an active sample can read them.
// ---------------------------------------------------------------------------
constexpr int GT_X = 32, GT_Y = kGateRows, GH = 4;
constexpr int GW = GT_X + 2 * GH, GHh = GT_Y + 2 * GH;

// Gradients of the three planes at one tile slot: (gx, gy) of lc in an
// 8-byte word and (gxU, gxV, gyU, gyV) in a 16-byte word, so a bilinear
// corner is two shared-memory loads and the U and V arithmetic runs on
// packed pairs straight from the loaded registers.
struct GateTile {
    float2 gl[GHh][GW];
    float4 guv[GHh][GW];
};

// U and V of one corner projected on the normal: (gxU*nx + gyU*ny,
// gxV*nx + gyV*ny), each lane rounded as the scalar expression.
__device__ __forceinline__ f32x2 projectUV(const float4 &g, f32x2 nx2, f32x2 ny2) {
    return add2(mul2(pk2(g.x, g.y), nx2), mul2(pk2(g.z, g.w), ny2));
}

// Gate of the active sample (x, y). INTERIOR: the tile and its halo lie
// inside the plane, so sample slots need no clamping.
template <bool INTERIOR>
__device__ __forceinline__ float gateAt(const GateTile &T, int x, int y, int x0, int y0, int w, int h) {
    auto sx = [&](int xx) { return (INTERIOR ? xx : iclamp(xx, 0, w - 1)) - x0 + GH; };
    auto sy = [&](int yy) { return (INTERIOR ? yy : iclamp(yy, 0, h - 1)) - y0 + GH; };
    float sxx = 0.0f, sxy = 0.0f, syy = 0.0f;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            const float2 g = T.gl[sy(y + dy)][sx(x + dx)];
            const float a = g.x, b = g.y;
            sxx += a * a; sxy += a * b; syy += b * b;
        }
    const float jsum = sxx + syy;
    if (jsum < 1e-10f)
        return 0.0f;
    const TensorDir dir = principalDirection(sxx, sxy, syy);
    const float nx = dir.nx, ny = dir.ny;
    // moments of (gY, gC) as packed pairs: sum, sum of squares, k-weighted sum
    const f32x2 nx2 = pk2(nx, nx), ny2 = pk2(ny, ny);
    f32x2 sum2 = pk2(0.0f, 0.0f), sq2 = sum2, mom2 = sum2;
    for (int k = -3; k <= 3; ++k) {
        const float px = (float)x + (float)k * nx;
        const float py = (float)y + (float)k * ny;
        const float fpx = floorf(px), fpy = floorf(py);
        const int rawX = (int)fpx, rawY = (int)fpy;
        const int bx0 = sx(rawX), bx1 = sx(rawX + 1);
        const int by0 = sy(rawY), by1 = sy(rawY + 1);
        const float fx = px - fpx, fy = py - fpy;
        const float2 A = T.gl[by0][bx0], B = T.gl[by0][bx1], C = T.gl[by1][bx0], D = T.gl[by1][bx1];
        float sY;
        {
            const float a = A.x * nx + A.y * ny, b = B.x * nx + B.y * ny;
            const float c = C.x * nx + C.y * ny, d = D.x * nx + D.y * ny;
            sY = a + (b - a) * fx + (c - a) * fy + (a - b - c + d) * fx * fy;
        }
        f32x2 sUV;
        {
            const f32x2 a = projectUV(T.guv[by0][bx0], nx2, ny2), b = projectUV(T.guv[by0][bx1], nx2, ny2);
            const f32x2 c = projectUV(T.guv[by1][bx0], nx2, ny2), d = projectUV(T.guv[by1][bx1], nx2, ny2);
            const f32x2 fx2 = pk2(fx, fx), fy2 = pk2(fy, fy);
            // a + (b - a) * fx + (c - a) * fy + (a - b - c + d) * fx * fy per lane
            sUV = add2(add2(add2(a, mul2(sub2(b, a), fx2)), mul2(sub2(c, a), fy2)),
                       mul2(mul2(add2(sub2(sub2(a, b), c), d), fx2), fy2));
        }
        float su, sv;
        up2(sUV, su, sv);
        const float gY = fabsf(sY);
        const float gC = sqrtf(su * su + sv * sv);
        const f32x2 g2 = pk2(gY, gC);
        const float kf = (float)k;
        sum2 = add2(sum2, g2);
        sq2 = add2(sq2, mul2(g2, g2));
        mom2 = add2(mom2, mul2(pk2(kf, kf), g2));
    }
    float sumY, sumC, sqY, sqC, momY, momC;
    up2(sum2, sumY, sumC);
    up2(sq2, sqY, sqC);
    up2(mom2, momY, momC);
    if (sumY < 1e-9f || sumC < 1e-9f)
        return 0.0f;
    const float partY = sumY * sumY / (sqY + 1e-12f);
    const float partC = sumC * sumC / (sqC + 1e-12f);
    const float ratio = partC / (partY + 1e-6f);
    const float dcent = fabsf(momY / sumY - momC / sumC);
    const float tw = sclamp((1.6f - ratio) / 0.4f, 0.0f, 1.0f);
    const float tp = sclamp((1.0f - dcent) / 0.5f, 0.0f, 1.0f);
    return (tw * tw * (3.0f - 2.0f * tw)) * (tp * tp * (3.0f - 2.0f * tp));
}

__global__ void __launch_bounds__(GT_X * 8)
k_gate(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    constexpr int SW = GW + 2, SH = GHh + 2;     // lc, U, V with the Sobel ring
    __shared__ float src[3][SH][SW];
    __shared__ GateTile T;
    __shared__ FrameJob sJob;
    __shared__ int sActive;
    static_assert(sizeof(src) >= GT_X * GT_Y * sizeof(uint16_t), "sample list fits the staged samples");
    // the active-sample list reuses the staged samples once the gradients exist
    uint16_t *sList = reinterpret_cast<uint16_t *>(&src[0][0][0]);
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    stageJob(jobs, f, sJob);
    const FrameJob &J = sJob;
    const int tile = blockIdx.x - tileStart[f];
    const int w = J.cw, h = J.ch;
    const int tilesX = (w + GT_X - 1) / GT_X;
    const int x0 = (tile % tilesX) * GT_X, y0 = (tile / tilesX) * GT_Y;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool dense = !J.sparse || J.gateDense ||
        (unsigned long long)J.counters[kCntActiveChroma] * 2ull >= (unsigned long long)w * h;
    if (!dense) {
        // a tile without active samples only stores the zeros of the gate plane
        bool any = false;
        const int x = x0 + tx;
        if (x < w)
            for (int y = y0 + ty; y < min(y0 + GT_Y, h); y += 8)
                any |= J.cmask[(size_t)y * w + x] != 0;
        if (!__syncthreads_or(any)) {
            if (x < w)
                for (int y = y0 + ty; y < min(y0 + GT_Y, h); y += 8)
                    J.ms[(size_t)y * w + x] = 0.0f;
            return;
        }
    }
    // samples at clamped positions of the tile, its halo and the Sobel ring
    const bool srcInterior = x0 >= GH + 1 && y0 >= GH + 1 && x0 + GT_X + GH + 1 <= w &&
                             y0 + GT_Y + GH + 1 <= h;
    for (int r = ty; r < SH; r += 8) {
        const int yy = srcInterior ? y0 - GH - 1 + r : iclamp(y0 - GH - 1 + r, 0, h - 1);
        for (int c = tx; c < SW; c += GT_X) {
            const int xx = srcInterior ? x0 - GH - 1 + c : iclamp(x0 - GH - 1 + c, 0, w - 1);
            const size_t o = (size_t)yy * w + xx;
            src[0][r][c] = ldf(J.lc + o);
            src[1][r][c] = ldf(J.U + o);
            src[2][r][c] = ldf(J.V + o);
        }
    }
    __syncthreads();
    // gradients at clamped positions of the tile and its halo (the dense
    // Sobel rows of the reference; the sparse reference computes the same
    // values wherever an active sample reads them)
    for (int r = ty; r < GHh; r += 8) {
        const int sr = (srcInterior ? y0 - GH + r : iclamp(y0 - GH + r, 0, h - 1)) - y0 + GH + 1;
        for (int c = tx; c < GW; c += GT_X) {
            const int sc = (srcInterior ? x0 - GH + c : iclamp(x0 - GH + c, 0, w - 1)) - x0 + GH + 1;
            float g[6];
#pragma unroll
            for (int p = 0; p < 3; ++p) {
                const float tl = src[p][sr - 1][sc - 1], t = src[p][sr - 1][sc], tr = src[p][sr - 1][sc + 1];
                const float l = src[p][sr][sc - 1], rr = src[p][sr][sc + 1];
                const float bl = src[p][sr + 1][sc - 1], b = src[p][sr + 1][sc], br = src[p][sr + 1][sc + 1];
                g[2 * p] = (tr + 2.0f * rr + br - tl - 2.0f * l - bl) * 0.125f;
                g[2 * p + 1] = (bl + 2.0f * b + br - tl - 2.0f * t - tr) * 0.125f;
            }
            T.gl[r][c] = make_float2(g[0], g[1]);
            T.guv[r][c] = make_float4(g[2], g[4], g[3], g[5]);
        }
    }
    // the tile's active samples, compacted so every thread takes a share
    // (inactive samples store the sparse plane's zeros here); the barrier also
    // ends the gradient pass's reads of the staged samples
    if (tx == 0 && ty == 0)
        sActive = 0;
    __syncthreads();
    const int x = x0 + tx;
    for (int r = ty; r < GT_Y; r += 8) {
        const int y = y0 + r;
        bool on = false;
        if (x < w && y < h) {
            const size_t o = (size_t)y * w + x;
            on = dense || J.cmask[o] != 0;
            if (!on)
                J.ms[o] = 0.0f;
        }
        const uint32_t ballot = __ballot_sync(0xffffffffu, on);
        int base = 0;
        if (tx == 0 && ballot)
            base = atomicAdd(&sActive, __popc(ballot));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (on)
            sList[base + __popc(ballot & ((1u << tx) - 1u))] = (uint16_t)(r * GT_X + tx);
    }
    __syncthreads();
    const bool interior = x0 >= GH && y0 >= GH && x0 + GT_X + GH <= w && y0 + GT_Y + GH <= h;
    const int count = sActive;
    for (int i = ty * GT_X + tx; i < count; i += GT_X * 8) {
        const int e = sList[i];
        const int sx = x0 + (e % GT_X), sy = y0 + e / GT_X;
        J.ms[(size_t)sy * w + sx] =
            interior ? gateAt<true>(T, sx, sy, x0, y0, w, h) : gateAt<false>(T, sx, sy, x0, y0, w, h);
    }
}

} // namespace lgcr_b200
