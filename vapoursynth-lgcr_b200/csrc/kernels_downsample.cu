// Downsample: 4:4:4 -> 4:2:0 chroma with a luma-guided correction, the
// reference's fourth filter (src/downsample.cpp).
//
// Per frame, three launches:
//   k_ds_rows   the base's horizontal polyphase pass (BaselineRing::ensureRow,
//               scalar form, downsample.cpp:176-226) for every source row:
//               one (U, V) pair per source row and output column;
//   k_ds_pixel  per output chroma sample: the vertical pass (makeRow,
//               140-168), then for strength > 0 the structure classification
//               (classify, 263-378) and the guided range/spatial averages
//               (accumulateGuided, 406-451) over a source tile staged in
//               shared memory; quality 0/1 store the final sample
//               (makeGuidedPixel, 465-509), quality 2 stores the base, the
//               gate and four candidates (generateCandidateRow, 524-569);
//   k_ds_score  quality 2: scores the candidates by re-upsampling them
//               bilinearly to the four source positions of the sample and
//               keeps the best (scoreCandidateRow, 577-651).
// All arithmetic is FP32 in the reference's order (the library is compiled
// without FMA contraction), with its clamped sample reads; quotients are
// IEEE divisions, or the reciprocal refinement equal to them on [1, 2^64)
// where the denominator is 1 plus a non-negative term.
#include "downsample.h"

namespace lgcr_b200 {

namespace {

struct DsDirection {
    float x, y;
};

// unit normals at 22.5 degree steps, the reference's direction table
// (downsample.cpp:239-248)
__constant__ DsDirection kDsDirections[8] = {
    {1.0f, 0.0f}, {0.9238795f, 0.3826834f}, {0.7071068f, 0.7071068f},
    {0.3826834f, 0.9238795f}, {0.0f, 1.0f}, {-0.3826834f, 0.9238795f},
    {-0.7071068f, 0.7071068f}, {-0.9238795f, 0.3826834f},
};

constexpr float kDsActivation = 1.0e-4f;     // guidedActivationThreshold
constexpr float kDsRangeScale2 = 2.25e-4f;   // accumulateGuided rangeScale2

// one output block: 32 x 8 chroma samples; its source tile covers every
// sample classify and accumulateGuided read (x in [2x - 4, 2x + 4], y in
// [2y - 4, 2y + 5] around output (x, y)), clamped like SourcePlane::at
constexpr int kDsBx = 32, kDsBy = 8;
constexpr int kDsHalo = 4;
constexpr int kDsTw = 2 * kDsBx + 2 * kDsHalo;        // 72
constexpr int kDsTh = 2 * kDsBy + 2 * kDsHalo;        // 24

template <int KIND>
__device__ __forceinline__ float dsLoad(const DownsampleJob &J, int plane, int x, int y) {
    x = iclamp(x, 0, J.W - 1);
    y = iclamp(y, 0, J.H - 1);
    const char *row = static_cast<const char *>(J.in[plane]) + (long long)y * J.inPitch[plane];
    const float off = plane == 0 ? 0.0f : J.chromaOffset;
    float raw;
    if (KIND == kU8)
        raw = (float)__ldg(reinterpret_cast<const unsigned char *>(row) + x);
    else if (KIND == kU16)
        raw = (float)__ldg(reinterpret_cast<const unsigned short *>(row) + x);
    else
        raw = __ldg(reinterpret_cast<const float *>(row) + x);
    return raw * J.inScale + off;
}

// OutputPlane::writeRow (downsample.cpp:113-127)
__device__ __forceinline__ void dsStore(const DownsampleJob &J, int plane, int x, int y, float v) {
    char *row = static_cast<char *>(J.out[plane]) + (long long)y * J.outPitch[plane];
    if (J.kind == kF32) {
        reinterpret_cast<float *>(row)[x] = v;
        return;
    }
    const int q = quantize(v, J.outScale, J.outOffset, J.maxCode);
    if (J.kind == kU8) reinterpret_cast<uint8_t *>(row)[x] = (uint8_t)q;
    else reinterpret_cast<uint16_t *>(row)[x] = (uint16_t)q;
}

// Shared source tile of one block: Y, U, V as floats, origin (ox, oy) in
// source coordinates.
struct DsTile {
    const float *y, *u, *v;
    int ox, oy;
    __device__ __forceinline__ int idx(int x, int yy) const { return (yy - oy) * kDsTw + (x - ox); }
    __device__ __forceinline__ float Y(int x, int yy) const { return y[idx(x, yy)]; }
    __device__ __forceinline__ float U(int x, int yy) const { return u[idx(x, yy)]; }
    __device__ __forceinline__ float V(int x, int yy) const { return v[idx(x, yy)]; }
};

// std::clamp's order of comparisons (NaN passes through)
__device__ __forceinline__ float dsClamp(float v, float lo, float hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}

struct DsStats {
    int primary, secondary;
    float secondaryMix, gate;
    bool isotropic;
};

// classify (downsample.cpp:263-378)
__device__ DsStats dsClassify(const DsTile &T, float centerX, float centerY, int quality) {
    const int ix = (int)floorf(centerX + 0.5f);
    const int iy = (int)floorf(centerY + 0.5f);
    float jxx = 0.0f, jxy = 0.0f, jyy = 0.0f, centerGx = 0.0f, centerGy = 0.0f;
    if (quality == 0) {
        const float tl = T.Y(ix - 1, iy - 1), tc = T.Y(ix, iy - 1), tr = T.Y(ix + 1, iy - 1);
        const float ml = T.Y(ix - 1, iy), mr = T.Y(ix + 1, iy);
        const float bl = T.Y(ix - 1, iy + 1), bc = T.Y(ix, iy + 1), br = T.Y(ix + 1, iy + 1);
        centerGx = (tr + 2.0f * mr + br - tl - 2.0f * ml - bl) * 0.125f;
        centerGy = (bl + 2.0f * bc + br - tl - 2.0f * tc - tr) * 0.125f;
        jxx = centerGx * centerGx;
        jxy = centerGx * centerGy;
        jyy = centerGy * centerGy;
    } else {
#pragma unroll
        for (int k = -1; k <= 1; ++k) {
            const float gx = 0.5f * (T.Y(ix + 1, iy + k) - T.Y(ix - 1, iy + k));
            const float gy = 0.5f * (T.Y(ix, iy + k + 1) - T.Y(ix, iy + k - 1));
            jxx += gx * gx;
            jxy += gx * gy;
            jyy += gy * gy;
            if (k == 0) {
                centerGx = gx;
                centerGy = gy;
            }
        }
    }
    DsStats st{0, 1, 0.0f, 0.0f, true};
    const float trace = jxx + jyy;
    if (trace < 1.0e-6f)
        return st;
    const float difference = jxx - jyy;
    const float discriminant2 = difference * difference + 4.0f * jxy * jxy;
    const float coherence2 = discriminant2 / (trace * trace + 1e-12f);

    float best = -1.0f, second = -1.0f;
    const int step = quality == 0 ? 2 : 1;
    for (int d = 0; d < 8; d += step) {
        const DsDirection n = kDsDirections[d];
        const float response = n.x * n.x * jxx + 2.0f * n.x * n.y * jxy + n.y * n.y * jyy;
        if (response > best) {
            second = best;
            st.secondary = st.primary;
            best = response;
            st.primary = d;
        } else if (response > second) {
            second = response;
            st.secondary = d;
        }
    }
    st.isotropic = coherence2 < (quality == 0 ? 0.20f : 0.10f);
    if (quality > 0 && best > 1e-12f) {
        const float adjacentAtExact = 0.8535534f;
        const float ratio = dsClamp(second / best, 0.0f, 1.0f);
        st.secondaryMix = 0.5f * dsClamp((ratio - adjacentAtExact) / (1.0f - adjacentAtExact),
                                         0.0f, 1.0f);
    }

    const float ugx = 0.5f * (T.U(ix + 1, iy) - T.U(ix - 1, iy));
    const float ugy = 0.5f * (T.U(ix, iy + 1) - T.U(ix, iy - 1));
    const float vgx = 0.5f * (T.V(ix + 1, iy) - T.V(ix - 1, iy));
    const float vgy = 0.5f * (T.V(ix, iy + 1) - T.V(ix, iy - 1));
    const float chromaEnergy = ugx * ugx + ugy * ugy + vgx * vgx + vgy * vgy;
    const DsDirection normal = kDsDirections[st.primary];
    const float un = ugx * normal.x + ugy * normal.y;
    const float vn = vgx * normal.x + vgy * normal.y;
    const float alignedEnergy = un * un + vn * vn;
    const int nsx = (int)lroundf(normal.x), nsy = (int)lroundf(normal.y);
    const float centerU = T.U(ix, iy), centerV = T.V(ix, iy);
    const float curvatureU = T.U(ix + nsx, iy + nsy) - 2.0f * centerU + T.U(ix - nsx, iy - nsy);
    const float curvatureV = T.V(ix + nsx, iy + nsy) - 2.0f * centerV + T.V(ix - nsx, iy - nsy);
    const float curvatureEnergy = curvatureU * curvatureU + curvatureV * curvatureV;
    const float sharpnessGate = curvatureEnergy / (curvatureEnergy + chromaEnergy + 1.0e-12f);

    const float lumaGate = trace / (trace + 3.0e-5f);
    const float confidenceGate = coherence2 / (coherence2 + 0.08f);
    const float chromaGate = chromaEnergy / (chromaEnergy + 2.0e-5f);
    const float directionGate = alignedEnergy / (chromaEnergy + 1.0e-12f);
    const float centerEnergy = centerGx * centerGx + centerGy * centerGy;
    const float positionGate = centerEnergy / (centerEnergy + 1.0e-5f);
    st.gate = dsClamp(lumaGate * confidenceGate * chromaGate * directionGate * positionGate *
                          sharpnessGate, 0.0f, 1.0f);
    if (quality == 0)
        st.gate *= 0.985f;
    else if (quality == 2)
        st.gate = (st.gate * 1.01f < 1.0f) ? st.gate * 1.01f : 1.0f;     // std::min
    if (sharpnessGate < (quality == 0 ? 0.20f : 0.12f))
        st.gate = 0.0f;
    return st;
}

struct DsEnvelope {
    DsDirection normal;
    int radius;
    float anisotropy;
    bool isotropic;
};

// spatialWeight (downsample.cpp:393-402); denominators are 1 plus
// non-negative terms of offsets within 4 samples
__device__ __forceinline__ float dsSpatial(const DsEnvelope &e, float dx, float dy) {
    const float radius2 = dx * dx + dy * dy;
    if (e.isotropic)
        return rcpInRange(1.0f + 0.42f * radius2);
    const float nd = dx * e.normal.x + dy * e.normal.y;
    const float td = -dx * e.normal.y + dy * e.normal.x;
    return rcpInRange(1.0f + (0.9f + e.anisotropy) * nd * nd + 0.16f * td * td);
}

// accumulateGuided (downsample.cpp:404-451): range- and spatially-weighted
// sums of U and V over the envelopes' common window, per envelope
template <int N>
__device__ __forceinline__ void dsAccumulate(const DsTile &T, float centerX, float centerY,
                                             const DsEnvelope (&env)[N], float (&aw)[N],
                                             float (&au)[N], float (&av)[N]) {
    int maxRadius = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        maxRadius = max(maxRadius, env[i].radius);
        aw[i] = au[i] = av[i] = 0.0f;
    }
    const int x0 = (int)ceilf(centerX - maxRadius), x1 = (int)floorf(centerX + maxRadius);
    const int y0 = (int)ceilf(centerY - maxRadius), y1 = (int)floorf(centerY + maxRadius);
    const int cx0 = (int)floorf(centerX), cy0 = (int)floorf(centerY);
    const float fx = centerX - cx0, fy = centerY - cy0;
    const float ya = T.Y(cx0, cy0), yb = T.Y(cx0 + 1, cy0);
    const float yc = T.Y(cx0, cy0 + 1), yd = T.Y(cx0 + 1, cy0 + 1);
    const float centerLuma = ya + (yb - ya) * fx + (yc - ya) * fy + (ya - yb - yc + yd) * fx * fy;
    for (int sy = y0; sy <= y1; ++sy) {
        for (int sx = x0; sx <= x1; ++sx) {
            const float dx = sx - centerX, dy = sy - centerY;
            const int o = T.idx(sx, sy);
            const float delta = T.y[o] - centerLuma;
            const float rangeWeight = kDsRangeScale2 / (kDsRangeScale2 + delta * delta);
            const float su = T.u[o], sv = T.v[o];
#pragma unroll
            for (int i = 0; i < N; ++i) {
                if (fabsf(dx) > env[i].radius || fabsf(dy) > env[i].radius)
                    continue;
                const float weight = rangeWeight * dsSpatial(env[i], dx, dy);
                aw[i] += weight;
                au[i] += weight * su;
                av[i] += weight * sv;
            }
        }
    }
}

// normalizedValue (downsample.cpp:459-461)
__device__ __forceinline__ float dsNorm(float sum, float weight, float fallback) {
    return weight > 1e-12f ? sum / weight : fallback;
}

// Horizontal pass of the base for every source row.
template <int KIND>
__global__ void __launch_bounds__(128) k_ds_rows(DownsampleJob J) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= J.cw)
        return;
    const int s = __ldg(J.hStart + x);
    const float *w = J.hW + (size_t)x * J.hSup;
    float su = 0.0f, sv = 0.0f;
    for (int tap = 0; tap < J.hSup; ++tap) {
        const float wt = __ldg(w + tap);
        su += wt * dsLoad<KIND>(J, 1, s + tap, y);
        sv += wt * dsLoad<KIND>(J, 2, s + tap, y);
    }
    J.rows[(size_t)y * J.cw + x] = make_float2(su, sv);
}

// Vertical pass, then (GUIDED) the guided correction or the candidates.
template <int KIND, bool GUIDED>
__global__ void __launch_bounds__(256) k_ds_pixel(DownsampleJob J) {
    __shared__ float sY[GUIDED ? kDsTw * kDsTh : 1], sU[GUIDED ? kDsTw * kDsTh : 1],
        sV[GUIDED ? kDsTw * kDsTh : 1];
    const int bx0 = blockIdx.x * kDsBx, by0 = blockIdx.y * kDsBy;
    const int x = bx0 + threadIdx.x, y = by0 + threadIdx.y;
    const bool inside = x < J.cw && y < J.ch;
    float bu = 0.0f, bv = 0.0f;
    if (inside) {
        const int s = __ldg(J.vStart + y);
        const float *w = J.vW + (size_t)y * J.vSup;
        for (int tap = 0; tap < J.vSup; ++tap) {
            const int sy = iclamp(s + tap, 0, J.H - 1);
            const float wt = __ldg(w + tap);
            const float2 r = J.rows[(size_t)sy * J.cw + x];
            bu += wt * r.x;
            bv += wt * r.y;
        }
    }
    if (!GUIDED) {
        if (inside) {
            dsStore(J, 0, x, y, bu);
            dsStore(J, 1, x, y, bv);
        }
        return;
    }
    DsTile T{sY, sU, sV, 2 * bx0 - kDsHalo, 2 * by0 - kDsHalo};
    for (int k = threadIdx.y * kDsBx + threadIdx.x; k < kDsTw * kDsTh; k += kDsBx * kDsBy) {
        const int sx = T.ox + k % kDsTw, sy = T.oy + k / kDsTw;
        sY[k] = dsLoad<KIND>(J, 0, sx, sy);
        sU[k] = dsLoad<KIND>(J, 1, sx, sy);
        sV[k] = dsLoad<KIND>(J, 2, sx, sy);
    }
    __syncthreads();
    if (!inside)
        return;
    const float centerX = 2.0f * x + 0.5f + J.shiftX;
    const float centerY = 2.0f * y + 0.5f + J.shiftY;
    const size_t o = (size_t)y * J.cw + x;
    if (J.quality < 2) {
        // makeGuidedPixel (downsample.cpp:465-509)
        const DsStats st = dsClassify(T, centerX, centerY, J.quality);
        float gu = bu, gv = bv, gate = st.gate;
        if (st.gate <= kDsActivation) {
            gate = 0.0f;
        } else if (J.quality == 0) {
            const DsEnvelope env[1] = {{kDsDirections[st.primary], 2, 1.8f, st.isotropic}};
            float aw[1], au[1], av[1];
            dsAccumulate<1>(T, centerX, centerY, env, aw, au, av);
            gu = dsNorm(au[0], aw[0], bu);
            gv = dsNorm(av[0], aw[0], bv);
        } else {
            const DsEnvelope env[2] = {{kDsDirections[st.primary], 3, 2.2f, st.isotropic},
                                       {kDsDirections[st.secondary], 3, 2.2f, st.isotropic}};
            float aw[2], au[2], av[2];
            dsAccumulate<2>(T, centerX, centerY, env, aw, au, av);
            const float u0 = dsNorm(au[0], aw[0], bu), v0 = dsNorm(av[0], aw[0], bv);
            const float u1 = dsNorm(au[1], aw[1], bu), v1 = dsNorm(av[1], aw[1], bv);
            gu = u0 + st.secondaryMix * (u1 - u0);
            gv = v0 + st.secondaryMix * (v1 - v0);
        }
        dsStore(J, 0, x, y, bu + J.strength * gate * (gu - bu));
        dsStore(J, 1, x, y, bv + J.strength * gate * (gv - bv));
        return;
    }
    // generateCandidateRow (downsample.cpp:524-569)
    const size_t plane = (size_t)J.cw * J.ch;
    float *C = J.cand + o;
    C[kDsBaseU * plane] = bu;
    C[kDsBaseV * plane] = bv;
    const DsStats st = dsClassify(T, centerX, centerY, 2);
    const float gate = st.gate > kDsActivation ? st.gate : 0.0f;
    C[kDsGate * plane] = gate;
    if (gate == 0.0f) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            C[(kDsCandU + c) * plane] = bu;
            C[(kDsCandV + c) * plane] = bv;
        }
        return;
    }
    const DsEnvelope env[5] = {
        {kDsDirections[st.primary], 3, 2.2f, st.isotropic},
        {kDsDirections[st.secondary], 3, 2.2f, st.isotropic},
        {kDsDirections[st.primary], 4, 2.7f, st.isotropic},
        {kDsDirections[st.secondary], 4, 2.7f, st.isotropic},
        {kDsDirections[st.primary], 4, 0.0f, true},
    };
    float aw[5], au[5], av[5];
    dsAccumulate<5>(T, centerX, centerY, env, aw, au, av);
    const float u0 = dsNorm(au[0], aw[0], bu), v0 = dsNorm(av[0], aw[0], bv);
    const float u1 = dsNorm(au[1], aw[1], bu), v1 = dsNorm(av[1], aw[1], bv);
    C[kDsCandU * plane] = u0 + st.secondaryMix * (u1 - u0);
    C[kDsCandV * plane] = v0 + st.secondaryMix * (v1 - v0);
#pragma unroll
    for (int c = 1; c < 4; ++c) {
        C[(kDsCandU + c) * plane] = dsNorm(au[c + 1], aw[c + 1], bu);
        C[(kDsCandV + c) * plane] = dsNorm(av[c + 1], aw[c + 1], bv);
    }
}

// scoreCandidateRow (downsample.cpp:571-651): re-upsample each candidate
// bilinearly to the sample's four source positions, keep the lowest
// edge-weighted squared error
template <int KIND>
__global__ void __launch_bounds__(256) k_ds_score(DownsampleJob J) {
    const int x = blockIdx.x * kDsBx + threadIdx.x, y = blockIdx.y * kDsBy + threadIdx.y;
    if (x >= J.cw || y >= J.ch)
        return;
    const size_t plane = (size_t)J.cw * J.ch;
    const float *C = J.cand;
    const size_t o = (size_t)y * J.cw + x;
    const float bu = C[kDsBaseU * plane + o], bv = C[kDsBaseV * plane + o];
    const float gate = C[kDsGate * plane + o];
    if (gate == 0.0f) {
        dsStore(J, 0, x, y, bu);
        dsStore(J, 1, x, y, bv);
        return;
    }
    float scores[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int hy = 2 * y; hy <= 2 * y + 1; ++hy) {
        for (int hx = 2 * x; hx <= 2 * x + 1; ++hx) {
            const float gx = 0.5f * (dsLoad<KIND>(J, 0, hx + 1, hy) - dsLoad<KIND>(J, 0, hx - 1, hy));
            const float gy = 0.5f * (dsLoad<KIND>(J, 0, hx, hy + 1) - dsLoad<KIND>(J, 0, hx, hy - 1));
            const float edge2 = gx * gx + gy * gy;
            const float edgeWeight = 0.125f + edge2 / (edge2 + 1.0e-5f);
            const float lowX = (hx - 0.5f - J.shiftX) * 0.5f;
            const float lowY = (hy - 0.5f - J.shiftY) * 0.5f;
            const float sourceU = dsLoad<KIND>(J, 1, hx, hy), sourceV = dsLoad<KIND>(J, 2, hx, hy);
            const int rawX0 = (int)floorf(lowX), rawY0 = (int)floorf(lowY);
            const int xa = iclamp(rawX0, 0, J.cw - 1), xb = iclamp(rawX0 + 1, 0, J.cw - 1);
            const int ra = iclamp(rawY0, 0, J.ch - 1), rb = iclamp(rawY0 + 1, 0, J.ch - 1);
            const float fx = lowX - rawX0, fy = lowY - rawY0;
            const float wts[4] = {(1.0f - fx) * (1.0f - fy), fx * (1.0f - fy), (1.0f - fx) * fy, fx * fy};
            const size_t at[4] = {(size_t)ra * J.cw + xa, (size_t)ra * J.cw + xb,
                                  (size_t)rb * J.cw + xa, (size_t)rb * J.cw + xb};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float ru = 0.0f, rv = 0.0f;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const float g = C[kDsGate * plane + at[k]];
                    float vu = C[kDsBaseU * plane + at[k]], vv = C[kDsBaseV * plane + at[k]];
                    vu += g * (C[(kDsCandU + c) * plane + at[k]] - vu);
                    vv += g * (C[(kDsCandV + c) * plane + at[k]] - vv);
                    ru += wts[k] * vu;
                    rv += wts[k] * vv;
                }
                const float du = ru - sourceU, dv = rv - sourceV;
                scores[c] += edgeWeight * (du * du + dv * dv);
            }
        }
    }
    int best = 0;
#pragma unroll
    for (int c = 1; c < 4; ++c)
        if (scores[c] < scores[best])
            best = c;
    dsStore(J, 0, x, y, bu + J.strength * gate * (C[(kDsCandU + best) * plane + o] - bu));
    dsStore(J, 1, x, y, bv + J.strength * gate * (C[(kDsCandV + best) * plane + o] - bv));
}

template <int KIND>
cudaError_t launchKind(const DownsampleJob &J, cudaStream_t s) {
    k_ds_rows<KIND><<<dim3((J.cw + 127) / 128, J.H), 128, 0, s>>>(J);
    const dim3 grid((J.cw + kDsBx - 1) / kDsBx, (J.ch + kDsBy - 1) / kDsBy), block(kDsBx, kDsBy);
    if (J.strength == 0.0f) {
        k_ds_pixel<KIND, false><<<grid, block, 0, s>>>(J);
    } else {
        k_ds_pixel<KIND, true><<<grid, block, 0, s>>>(J);
        if (J.quality == 2)
            k_ds_score<KIND><<<grid, block, 0, s>>>(J);
    }
    return cudaGetLastError();
}

} // namespace

cudaError_t launchDownsample(const DownsampleJob &J, cudaStream_t s) {
    if (J.kind == kU8)
        return launchKind<kU8>(J, s);
    if (J.kind == kU16)
        return launchKind<kU16>(J, s);
    return launchKind<kF32>(J, s);
}

} // namespace lgcr_b200
