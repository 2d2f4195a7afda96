// Sharpen: gated bilateral unsharp mask over a 5x5 window, the reference's
// second filter (sharpenGetFrame src/plugin.cpp:14-76, sharpenPlane
// src/algos.cpp:595-659).
//
// Per sample: the window's guide range max|g - L0| and sample hull, a sigma
// floor from the median of the four neighbour differences, then 24 taps with
// n = sp(i, j) * sim(dL), out = c0 + alpha * sum(n * (c0 - s)) / sum(n),
// clamped to the hull +- ar. Luma guides itself; subsampled chroma is guided
// by the footprint-average map of the already sharpened luma (lc) with the
// reference point bilinear on that luma at the sample's left-sited position;
// 4:4:4 chroma guides itself.
//
// Layout: one block sharpens a 32 x 8 tile of one plane. The source tile and
// a 2-sample halo (clamped coordinates, as the reference's Plane::at) are
// converted from the raw input into shared memory once; for guided chroma
// the lc tile with its halo is built in shared memory from the sharpened
// luma. All float arithmetic follows the reference's order (the library is
// compiled without FMA contraction); the 1/(1 + ...) quotients use the
// reciprocal refinement that equals the IEEE quotient on [1, 2^64).
#include "sharpen.h"

namespace lgcr_b200 {

namespace {

constexpr int kTx = 32, kTy = 8, kHalo = 2;
constexpr int kLx = kTx + 2 * kHalo, kLy = kTy + 2 * kHalo;

template <int KIND>
__device__ __forceinline__ float loadSample(const SharpenJob &J, int plane, int x, int y) {
    const char *row = static_cast<const char *>(J.in[plane]) + (long long)y * J.inPitch[plane];
    const double off = (plane == 0 || KIND == kF32) ? 0.0 : J.cOffset;
    if (KIND == kU8)
        return (float)((double)__ldg(reinterpret_cast<const unsigned char *>(row) + x) * J.yScale + off);
    if (KIND == kU16)
        return (float)((double)__ldg(reinterpret_cast<const unsigned short *>(row) + x) * J.yScale + off);
    return __ldg(reinterpret_cast<const float *>(row) + x) + 0.0f;   // s * 1.0 + 0.0
}

__device__ __forceinline__ void storeSample(const SharpenJob &J, int plane, int x, int y, float v) {
    char *row = static_cast<char *>(J.out[plane]) + (long long)y * J.outPitch[plane];
    if (J.kind == kF32) {
        reinterpret_cast<float *>(row)[x] = v + 0.0f;          // s * 1.0 + 0.0
        return;
    }
    const int q = quantize(v, J.qScale, plane == 0 ? 0.0f : J.qOffC, J.maxCode);
    if (J.kind == kU8) reinterpret_cast<uint8_t *>(row)[x] = (uint8_t)q;
    else reinterpret_cast<uint16_t *>(row)[x] = (uint16_t)q;
}

// reference bilinear (src/lgcr.h:467-475) at a position given in double
__device__ __forceinline__ float bilinearD(const float *p, int w, int h, double x, double y) {
    const double flx = floor(x), fly = floor(y);
    const int x0 = (int)flx, y0 = (int)fly;
    const float fx = (float)(x - (double)x0);
    const float fy = (float)(y - (double)y0);
    const int xa = iclamp(x0, 0, w - 1), xb = iclamp(x0 + 1, 0, w - 1);
    const int ya = iclamp(y0, 0, h - 1), yb = iclamp(y0 + 1, 0, h - 1);
    const float a = ldf(p + (size_t)ya * w + xa), b = ldf(p + (size_t)ya * w + xb);
    const float c = ldf(p + (size_t)yb * w + xa), d = ldf(p + (size_t)yb * w + xb);
    return a + (b - a) * fx + (c - a) * fy + (a - b - c + d) * fx * fy;
}

// One sample of sharpenPlane. S: source tile, G: guide tile (S itself when
// self-guided), both kLx wide with the sample at (tx + 2, ty + 2).
__device__ __forceinline__ float sharpenSample(const SharpenJob &J, const float *S, const float *G,
                                               int tx, int ty, float L0) {
    const int c = (ty + kHalo) * kLx + tx + kHalo;
    const float c0 = S[c];
    float maxAbsDL = 0.0f, hullMin = 1e30f, hullMax = -1e30f;
#pragma unroll
    for (int j = -2; j <= 2; ++j)
#pragma unroll
        for (int i = -2; i <= 2; ++i) {
            const int o = c + j * kLx + i;
            maxAbsDL = smax(maxAbsDL, fabsf(G[o] - L0));
            hullMin = smin(hullMin, S[o]);
            hullMax = smax(hullMax, S[o]);
        }
    // median of the four neighbour differences: the middle two of a sorted
    // four are max(min pair) and min(max pair)
    const float d0 = fabsf(S[c + 1] - c0), d1 = fabsf(S[c - 1] - c0);
    const float d2 = fabsf(S[c + kLx] - c0), d3 = fabsf(S[c - kLx] - c0);
    const float lo = smax(smin(d0, d1), smin(d2, d3));
    const float hi = smin(smax(d0, d1), smax(d2, d3));
    const float slopeMed = (lo + hi) * 0.5f;
    const float sig = smax(smax(J.sigma, J.sratio * maxAbsDL), 3.0f * slopeMed);
    const float invS2 = 1.0f / (sig * sig);
    // spatial bump 1/(1 + r^2/g^2) for r^2 = 1, 2, 4, 5, 8
    float sp[9];
#pragma unroll
    for (int r2 = 1; r2 <= 8; ++r2)
        sp[r2] = rcpAtLeastOne(1.0f + (float)r2 * J.invG2);
    float hp = 0.0f, wsum = 0.0f;
#pragma unroll
    for (int j = -2; j <= 2; ++j)
#pragma unroll
        for (int i = -2; i <= 2; ++i) {
            if (i == 0 && j == 0)
                continue;
            const int o = c + j * kLx + i;
            const float dL = G[o] - L0;
            const float sim = rcpAtLeastOne(1.0f + dL * dL * invS2);
            const float n = sp[i * i + j * j] * sim;
            hp += n * (c0 - S[o]);
            wsum += n;
        }
    float out = c0;
    if (wsum > 1e-6f)
        out = c0 + J.alpha * hp / wsum;
    if (J.clampHull)
        out = sclamp(out, hullMin - J.margin, hullMax + J.margin);
    return out;
}

// Self-guided planes: luma (blockIdx.z == 0) and, for 4:4:4, both chroma
// planes (blockIdx.z == 1, 2). Luma also writes the float sharpened plane
// the chroma guide reads.
template <int KIND>
__global__ void __launch_bounds__(kTx * kTy)
k_sharpen_self(const SharpenJob J) {
    __shared__ float S[kLx * kLy];
    const int plane = blockIdx.z;
    const int w = plane == 0 ? J.sw : J.cw, h = plane == 0 ? J.sh : J.ch;
    const int x0 = blockIdx.x * kTx, y0 = blockIdx.y * kTy;
    if (x0 >= w || y0 >= h)
        return;
    for (int k = threadIdx.y * kTx + threadIdx.x; k < kLx * kLy; k += kTx * kTy) {
        const int lx = k % kLx, ly = k / kLx;
        S[k] = loadSample<KIND>(J, plane, iclamp(x0 + lx - kHalo, 0, w - 1),
                                iclamp(y0 + ly - kHalo, 0, h - 1));
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= w || y >= h)
        return;
    const int c = (threadIdx.y + kHalo) * kLx + threadIdx.x + kHalo;
    const float v = sharpenSample(J, S, S, threadIdx.x, threadIdx.y, S[c]);
    if (plane == 0 && J.Ys)
        J.Ys[(size_t)y * J.sw + x] = v;
    storeSample(J, plane, x, y, v);
}

// Subsampled chroma guided by the sharpened luma: blockIdx.z = 0 (U), 1 (V).
template <int KIND>
__global__ void __launch_bounds__(kTx * kTy)
k_sharpen_chroma(const SharpenJob J) {
    __shared__ float S[kLx * kLy];
    __shared__ float G[kLx * kLy];
    const int plane = 1 + blockIdx.z;
    const int w = J.cw, h = J.ch;
    const int x0 = blockIdx.x * kTx, y0 = blockIdx.y * kTy;
    if (x0 >= w || y0 >= h)
        return;
    for (int k = threadIdx.y * kTx + threadIdx.x; k < kLx * kLy; k += kTx * kTy) {
        const int lx = k % kLx, ly = k / kLx;
        const int cx = iclamp(x0 + lx - kHalo, 0, w - 1), cy = iclamp(y0 + ly - kHalo, 0, h - 1);
        S[k] = loadSample<KIND>(J, plane, cx, cy);
        // lc: raster-order double sum of the sharpened luma over the
        // sample's footprint (buildLcMap src/maps.cpp:425-499)
        const int xb = __ldg(J.lcXb + cx), xe = __ldg(J.lcXe + cx);
        const int yb = __ldg(J.lcYb + cy), ye = __ldg(J.lcYe + cy);
        double sum = 0.0;
        for (int yy = yb; yy < ye; ++yy)
            for (int xx = xb; xx < xe; ++xx)
                sum += (double)ldf(J.Ys + (size_t)yy * J.sw + xx);
        G[k] = (float)(sum / ((double)(xe - xb) * (double)(ye - yb)));
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= w || y >= h)
        return;
    const float L0 = bilinearD(J.Ys, J.sw, J.sh, ((double)x + 0.5) * J.rw - 0.5 + J.shiftX,
                               ((double)y + 0.5) * J.rh - 0.5 + J.shiftY);
    storeSample(J, plane, x, y, sharpenSample(J, S, G, threadIdx.x, threadIdx.y, L0));
}

template <int KIND>
cudaError_t launchKind(const SharpenJob &J, cudaStream_t s) {
    const dim3 block(kTx, kTy);
    const bool guided = J.guided != 0;
    const int planes = guided ? 1 : 3;
    const int gw = guided ? J.sw : max(J.sw, J.cw), gh = guided ? J.sh : max(J.sh, J.ch);
    k_sharpen_self<KIND><<<dim3((gw + kTx - 1) / kTx, (gh + kTy - 1) / kTy, planes), block, 0, s>>>(J);
    if (guided)
        k_sharpen_chroma<KIND><<<dim3((J.cw + kTx - 1) / kTx, (J.ch + kTy - 1) / kTy, 2), block, 0, s>>>(J);
    return cudaGetLastError();
}

} // namespace

cudaError_t launchSharpen(const SharpenJob &J, cudaStream_t s) {
    switch (J.kind) {
    case kU8: return launchKind<kU8>(J, s);
    case kU16: return launchKind<kU16>(J, s);
    default: return launchKind<kF32>(J, s);
    }
}

} // namespace lgcr_b200
