// algo 6 (constrained detail transfer) and algo 4 (selector) stages.
//   k_yc              buildYcFilteredMaps + median3 consensus    src/maps.cpp:529-680,
//                                                                src/algos.cpp:813-815
//   k_affine          buildAffineMaps: 5x5 hull + 16 moments     src/algos.cpp:1026-1137,
//                     (sparse: direct sums, *1/n; dense: /n)     src/algos.cpp:1382-1526
//   k_detail_plain    plain reconstruct of D(Y) minus Y          src/algos.cpp:1528-1585
//   k_detail_nyq      dyadic [1/4,1/2,1/4] Nyquist passes        src/algos.cpp:1139-1364
//   k_detail_resize_* detail to output size                      src/algos.cpp:1366-1380
//   k_detail_transfer detailTransferImpl                         src/algos.cpp:1587-1698
//   k_lgf             buildLGFPair moments + ms fade             src/algos.cpp:300-448,
//                                                                src/plugin.cpp:418-425,543-551
//   k_roi             selector ROI marking                       src/plugin.cpp:496-531
//   k_blend           blendSelector / blendSelectorCompressed    src/algos.cpp:453-593
// Window moments are FP64 sums of exact float products in raster order.
#include "kernels.cuh"
#include "plain.cuh"

namespace lgcr_b200 {

__device__ __forceinline__ float median3f(float a, float b, float c) {
    const float mn = smin(smin(a, b), c);
    const float mx = smax(smax(a, b), c);
    return a + b + c - mn - mx;
}

// separable candidate D(Y) at one chroma sample: H pass (double acc, float
// store) on each needed luma row, then V pass (double acc).
__device__ __forceinline__ float candidateAt(const FrameJob &J, const WeightView &th,
                                             const WeightView &tv, int cx, int cy) {
    const int sv = __ldg(tv.start + cy);
    const float *wv = tv.w + (size_t)cy * tv.sup;
    const int shs = __ldg(th.start + cx);
    const float *wh = th.w + (size_t)cx * th.sup;
    double acc = 0.0;
    for (int j = 0; j < tv.sup; ++j) {
        const float *row = J.Y + (size_t)iclamp(sv + j, 0, J.sh - 1) * J.sw;
        double hv = 0.0;
        for (int i = 0; i < th.sup; ++i)
            hv = fma((double)__ldg(wh + i), (double)ldf(row + iclamp(shs + i, 0, J.sw - 1)), hv);
        acc = fma((double)__ldg(wv + j), (double)(float)hv, acc);
    }
    return (float)acc;
}

__global__ void k_yc_h(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int cx, cy;
    tile32x8(blockIdx.x - tileStart[f], J.cw, cx, cy);
    if (cx >= J.cw || cy >= J.ch)
        return;
    const size_t o = (size_t)cy * J.cw + cx;
    const float y1 = candidateAt(J, J.ycH1, J.ycV1, cx, cy);
    const float y2 = candidateAt(J, J.ycH2, J.ycV2, cx, cy);
    J.yc1[o] = y1;
    J.yc2[o] = y2;
    const size_t C = (size_t)J.cw * J.ch;
    J.aff[8 * C + o] = median3f(ldf(J.lc + o), y1, y2);   // degraded luma consensus
}

// The same candidates for a 32 x 32 tile of chroma samples: the horizontal
// sums of every luma row the tile reads go to shared memory once (per
// candidate), then each sample runs its vertical pass from there. Same
// operands and order as candidateAt. Tap supports up to 8.
__device__ __forceinline__ float ycHorizontal(const FrameJob &J, const WeightView &th, int cx, int row,
                                              const double (&w)[8], int s0) {
    const float *lrow = J.Y + (size_t)row * J.sw;
    double hv = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        if (i < th.sup)
            hv = fma(w[i], (double)ldf(lrow + iclamp(s0 + i, 0, J.sw - 1)), hv);
    return (float)hv;
}

__device__ __forceinline__ float ycVertical(const FrameJob &J, const WeightView &tv, int cy,
                                            const float (*sH)[32], int lo, int lx) {
    const int sv = __ldg(tv.start + cy);
    const float *wv = tv.w + (size_t)cy * tv.sup;
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j)
        if (j < tv.sup)
            acc = fma((double)__ldg(wv + j), (double)sH[iclamp(sv + j, 0, J.sh - 1) - lo][lx], acc);
    return (float)acc;
}

__global__ void __launch_bounds__(256)
k_yc_tiled(LGCR_STAGE_ARGS) {
    __shared__ float sH1[kYcRows][32];
    __shared__ float sH2[kYcRows][32];
    __shared__ FrameJob sJob;
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    stageJob(jobs, f, sJob);
    const FrameJob &J = sJob;
    const int tile = blockIdx.x - tileStart[f];
    const int tilesX = (J.cw + kYcTile - 1) / kYcTile;
    const int cx0 = (tile % tilesX) * kYcTile, cy0 = (tile / tilesX) * kYcTile;
    const int cyLast = min(cy0 + kYcTile, J.ch) - 1;
    const int lx = threadIdx.x;
    const int cx = cx0 + lx;
    const int cxc = min(cx, J.cw - 1);
    const int lo1 = iclamp(__ldg(J.ycV1.start + cy0), 0, J.sh - 1);
    const int hi1 = iclamp(__ldg(J.ycV1.start + cyLast) + J.ycV1.sup - 1, 0, J.sh - 1);
    const int lo2 = iclamp(__ldg(J.ycV2.start + cy0), 0, J.sh - 1);
    const int hi2 = iclamp(__ldg(J.ycV2.start + cyLast) + J.ycV2.sup - 1, 0, J.sh - 1);
    {
        double w1[8], w2[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            w1[i] = i < J.ycH1.sup ? (double)__ldg(J.ycH1.w + (size_t)cxc * J.ycH1.sup + i) : 0.0;
            w2[i] = i < J.ycH2.sup ? (double)__ldg(J.ycH2.w + (size_t)cxc * J.ycH2.sup + i) : 0.0;
        }
        const int s1 = __ldg(J.ycH1.start + cxc), s2 = __ldg(J.ycH2.start + cxc);
        for (int r = threadIdx.y; r <= hi1 - lo1; r += blockDim.y)
            sH1[r][lx] = ycHorizontal(J, J.ycH1, cxc, lo1 + r, w1, s1);
        for (int r = threadIdx.y; r <= hi2 - lo2; r += blockDim.y)
            sH2[r][lx] = ycHorizontal(J, J.ycH2, cxc, lo2 + r, w2, s2);
    }
    __syncthreads();
    if (cx >= J.cw)
        return;
    const size_t C = (size_t)J.cw * J.ch;
    for (int k = threadIdx.y; cy0 + k <= cyLast; k += blockDim.y) {
        const int cy = cy0 + k;
        const size_t o = (size_t)cy * J.cw + cx;
        const float y1 = ycVertical(J, J.ycV1, cy, sH1, lo1, lx);
        const float y2 = ycVertical(J, J.ycV2, cy, sH2, lo2, lx);
        J.yc1[o] = y1;
        J.yc2[o] = y2;
        J.aff[8 * C + o] = median3f(ldf(J.lc + o), y1, y2);   // degraded luma consensus
    }
}

// 5x5 affine statistics of one chroma sample (buildAffineMaps,
// src/algos.cpp:1026-1526).
__device__ __forceinline__ bool affineSparse(const FrameJob &J) {
    return J.sparse && (unsigned long long)J.counters[kCntActiveChroma] * 2ull <
                           (unsigned long long)J.cw * J.ch;
}

__device__ __forceinline__ void affineSample(const FrameJob &J, int x, int y, bool sparseRoi) {
    const int w = J.cw, h = J.ch;
    const size_t o = (size_t)y * w + x;
    const int top = max(0, y - 2), bottom = min(h - 1, y + 2);
    const int left = max(0, x - 2), right = min(w - 1, x + 2);
    const float *yc[3] = { J.lc, J.yc1, J.yc2 };
    double s[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) s[k] = 0.0;
    float mnU = ldf(J.U + (size_t)top * w + left), mxU = mnU;
    float mnV = ldf(J.V + (size_t)top * w + left), mxV = mnV;
    auto tap = [&](size_t q) {
        const float uf = ldf(J.U + q), vf = ldf(J.V + q);
        const double u = uf, v = vf;
        s[0] += u; s[1] += u * u; s[2] += v; s[3] += v * v;
        mnU = smin(mnU, uf); mxU = smax(mxU, uf);
        mnV = smin(mnV, vf); mxV = smax(mxV, vf);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double ly = ldf(yc[k] + q);
            const int b = 4 + 4 * k;
            s[b] += ly; s[b + 1] += ly * ly; s[b + 2] += ly * u; s[b + 3] += ly * v;
        }
    };
    if (bottom - top == 4 && right - left == 4) {
        // full 5x5 window: fixed offsets from its first sample
        const size_t q0 = (size_t)top * w + left;
#pragma unroll
        for (int dy = 0; dy < 5; ++dy)
#pragma unroll
            for (int dx = 0; dx < 5; ++dx)
                tap(q0 + (size_t)dy * w + dx);
    } else {
        for (int py = top; py <= bottom; ++py)
            for (int px = left; px <= right; ++px)
                tap((size_t)py * w + px);
    }
    const int n = (right - left + 1) * (bottom - top + 1);
    const double eps = J.lgfEps;
    const double epsSig = J.epsSig;
    const double inv = 1.0 / n;
    auto mean = [&](double sum) { return sparseRoi ? sum * inv : sum / n; };
    const double meanU = mean(s[0]), meanV = mean(s[2]);
    const double varU = smax(0.0, mean(s[1]) - meanU * meanU);
    const double varV = smax(0.0, mean(s[3]) - meanV * meanV);
    double q[3], aU[3], aV[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int b = 4 + 4 * k;
        const double meanY = mean(s[b]);
        const double varY = smax(0.0, mean(s[b + 1]) - meanY * meanY);
        const double covU = mean(s[b + 2]) - meanY * meanU;
        const double covV = mean(s[b + 3]) - meanY * meanV;
        aU[k] = sclamp(covU / (varY + eps), -16.0, 16.0);
        aV[k] = sclamp(covV / (varY + eps), -16.0, 16.0);
        q[k] = sclamp((covU * covU + covV * covV) / ((varY + eps) * (varU + varV + eps)), 0.0, 1.0);
    }
    const size_t C = (size_t)w * h;
    const float slopeU = median3f((float)aU[0], (float)aU[1], (float)aU[2]);
    const float slopeV = median3f((float)aV[0], (float)aV[1], (float)aV[2]);
    const double qmax = smax(smax(q[0], q[1]), q[2]);
    const double qmin = smin(smin(q[0], q[1]), q[2]);
    const double stability = qmax > 1e-9 ? qmin / qmax : 0.0;
    const double chromaSignal = (varU + varV) / (varU + varV + epsSig);
    const float gain = (float)(((q[0] + q[1] + q[2]) / 3.0) * stability * chromaSignal);
    // interleaved maps: (aU, aV, g, rng) then (mnU, mxU, mnV, mxV) per sample
    reinterpret_cast<float4 *>(J.aff)[o] = make_float4(slopeU, slopeV, gain, smax(mxU - mnU, mxV - mnV));
    reinterpret_cast<float4 *>(J.aff + 4 * C)[o] = make_float4(mnU, mxU, mnV, mxV);
}

// Tiled form (frames without a chroma work list): active samples when sparse.
__global__ void __launch_bounds__(256, 3)
k_affine(LGCR_STAGE_ARGS) {
    __shared__ FrameJob sJob;
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    stageJob(jobs, f, sJob);
    const FrameJob &J = sJob;
    int x, y;
    tile32x8(blockIdx.x - tileStart[f], J.cw, x, y);
    if (x >= J.cw || y >= J.ch)
        return;
    const bool sparseRoi = affineSparse(J);
    if (sparseRoi && J.cmask[(size_t)y * J.cw + x] == 0)
        return;
    affineSample(J, x, y, sparseRoi);
}

// Sparse frames: a persistent grid walks the compacted list of active chroma
// samples (every sample, in raster order, once the frame counts as dense),
// so no lane idles on an inactive sample.
constexpr int kAffineMaxFrames = 1024;

__global__ void __launch_bounds__(256, 3)
k_affine_list(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    __shared__ unsigned long long pre[kAffineMaxFrames + 1];
    for (int chunk = 0; chunk < njobs; chunk += kAffineMaxFrames) {
        const int n = min(kAffineMaxFrames, njobs - chunk);
        if (threadIdx.x == 0) {
            unsigned long long acc = 0;
            for (int i = 0; i < n; ++i) {
                pre[i] = acc;
                const FrameJob &J = jobs[chunk + i];
                if (J.chromaList)
                    acc += affineSparse(J) ? J.counters[kCntActiveChroma]
                                           : (unsigned long long)J.cw * J.ch;
            }
            pre[n] = acc;
        }
        __syncthreads();
        const unsigned long long total = pre[n];
        for (unsigned long long w = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; w < total;
             w += (unsigned long long)gridDim.x * blockDim.x) {
            int lo = 0, hi = n - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (pre[mid] <= w) lo = mid; else hi = mid - 1;
            }
            const FrameJob &J = jobs[chunk + lo];
            const unsigned long long k = w - pre[lo];
            const bool sparseRoi = affineSparse(J);
            int x, y;
            if (sparseRoi) {
                const uint32_t e = __ldg(J.chromaList + k);
                x = (int)(e & 0xffffu);
                y = (int)(e >> 16);
            } else {
                y = (int)(k / (unsigned long long)J.cw);
                x = (int)(k - (unsigned long long)y * J.cw);
            }
            affineSample(J, x, y, sparseRoi);
        }
        __syncthreads();
    }
}

// Horizontal pass of the degraded-luma reconstruction (separable kernels):
// per (source luma column, chroma row) the double sum over the active taps
// rounded to float, and the row's extrema (plainChromaSeparable with one
// plane, src/recon.cpp:1178-1271).
__global__ void __launch_bounds__(256)
k_detail_hpass(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int x, sy;
    tile32x8(blockIdx.x - tileStart[f], J.sw, x, sy);
    if (x >= J.sw || sy >= J.ch)
        return;
    const AxisView &ax = J.sax;
    const int tx0 = __ldg(ax.start + x);
    const double *wx = ax.wd + (size_t)x * ax.sup;
    const uint8_t *amx = ax.am + (size_t)x * ax.sup;
    const float *row = J.aff + 8 * (size_t)J.cw * J.ch + (size_t)sy * J.cw;
    double h = 0.0;
    float mn = 1e30f, mx = -1e30f;
    for (int i = 0; i < ax.sup; ++i) {
        if (__ldg(amx + i) == 0)
            continue;
        const float a = ldf(row + iclamp(tx0 + i, 0, J.cw - 1));
        h = fma(__ldg(wx + i), (double)a, h);
        mn = runMin(mn, a); mx = runMax(mx, a);
    }
    reinterpret_cast<float4 *>(J.dTab)[(size_t)sy * J.sw + x] = make_float4((float)h, mn, mx, 0.0f);
}

// detail = Y - plain(D(Y)) on the source luma grid.
__global__ void k_detail_plain(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int x, y;
    tile32x8(blockIdx.x - tileStart[f], J.sw, x, y);
    if (x >= J.sw || y >= J.sh)
        return;
    const size_t o = (size_t)y * J.sw + x;
    if (J.dTab) {
        // vertical pass over the horizontal table
        const AxisView &ax = J.sax, &ay = J.say;
        const int ty0 = __ldg(ay.start + y);
        const double *wy = ay.wd + (size_t)y * ay.sup;
        const uint8_t *amy = ay.am + (size_t)y * ay.sup;
        double v = 0.0;
        float mn = 1e30f, mx = -1e30f;
#pragma unroll 8
        for (int j = 0; j < ay.sup; ++j) {
            if (__ldg(amy + j) == 0)
                continue;
            const int sy = iclamp(ty0 + j, 0, J.ch - 1);
            const float4 t = __ldg(reinterpret_cast<const float4 *>(J.dTab) + (size_t)sy * J.sw + x);
            v = fma(__ldg(wy + j), (double)t.x, v);
            mn = runMin(mn, t.y); mx = runMax(mx, t.z);
        }
        const double ws = (double)__ldg(ax.wsum + x) * (double)__ldg(ay.wsum + y);
        const double wa = (double)__ldg(ax.wabs + x) * (double)__ldg(ay.wabs + y);
        const float *dgl = J.aff + 8 * (size_t)J.cw * J.ch;
        if (ws > 1e-6 && ws >= 0.05 * wa)
            v /= ws;
        else
            v = bilinearAt(dgl, J.cw, J.ch, __ldg(ax.pos + x), __ldg(ay.pos + y));
        if (J.clampHull)
            v = sclamp(v, (double)(mn - J.margin), (double)(mx + J.margin));
        J.detailTmp[o] = ldf(J.Y + o) - (float)v;
        return;
    }
    PlainCtx c = chromaPlainCtx(J);
    c.p0 = J.aff + 8 * (size_t)J.cw * J.ch;
    c.p1 = nullptr;
    c.ax = J.sax;
    c.ay = J.say;
    c.rad = J.srad;
    c.invWxC = J.sinvWxC;
    c.invWyC = J.sinvWyC;
    c.noClampX = J.sNoClampX;
    c.noClampY = J.sNoClampY;
    c.uv = nullptr;
    float r, unused;
    plainAt(c, x, y, r, unused);
    J.detailTmp[o] = ldf(J.Y + o) - r;
}

// ---------------------------------------------------------------------------
// Fused detail map (separable kernels, supports up to 8 taps): the horizontal
// pass of the degraded luma into shared memory, the vertical pass and
// detail = Y - plain(D(Y)), then the Nyquist passes (at most one per axis:
// chroma ratios are at most 2) on a 32-wide tile with a one-sample halo; the
// block writes the 30-column interior of J.detailRows rows (62, or 30 when
// the taller tile's chroma rows do not fit) to the detail plane. Samples sit at
// clamped coordinates, so at the plane borders the halo holds exactly the
// clamped neighbours the reference's passes read (buildDetailMap,
// src/algos.cpp:1528-1585, with suppressSourceNyquist 1303-1364).
// ---------------------------------------------------------------------------
struct DetailRows {
    double w[kDetailRowsTall + 2][8];
    int ty0[kDetailRowsTall + 2], r[kDetailRowsTall + 2];
    uint32_t act[kDetailRowsTall + 2];
    float wsum[kDetailRowsTall + 2], wabs[kDetailRowsTall + 2], pos[kDetailRowsTall + 2];
};

__device__ __forceinline__ uint32_t activityBits(const uint8_t *am, int n) {
    uint32_t m = 0;
    for (int i = 0; i < n; ++i)
        m |= (__ldg(am + i) != 0 ? 1u : 0u) << i;
    return m;
}

template <bool NOCLAMP>
__device__ __forceinline__ void detailEntry(const float *row, int cw, int tx0, const double (&w)[8],
                                            uint32_t act, double &hOut, float2 &ext) {
    double acc = 0.0;
    float lo = 1e30f, hi = -1e30f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (!((act >> i) & 1u))
            continue;
        const float a = ldf(row + (NOCLAMP ? tx0 + i : iclamp(tx0 + i, 0, cw - 1)));
        acc = fma(w[i], (double)a, acc);
        lo = runMin(lo, a);
        hi = runMax(hi, a);
    }
    hOut = (double)(float)acc;
    ext = make_float2(lo, hi);
}

template <bool NOCLAMP>
__device__ __forceinline__ double detailVertical(const DetailRows &R, const double (*sH)[32],
                                                 const float2 (*sE)[32], int k, int lx, int syLo,
                                                 int ch, float &mn, float &mx) {
    const int ty0 = R.ty0[k];
    const uint32_t act = R.act[k];
    double v = 0.0;
    float lo = 1e30f, hi = -1e30f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (!((act >> j) & 1u))
            continue;
        const int r = (NOCLAMP ? ty0 + j : iclamp(ty0 + j, 0, ch - 1)) - syLo;
        v = fma(R.w[k][j], sH[r][lx], v);
        const float2 e = sE[r][lx];
        lo = runMin(lo, e.x);
        hi = runMax(hi, e.y);
    }
    mn = lo;
    mx = hi;
    return v;
}

__global__ void __launch_bounds__(256)
k_detail_map(LGCR_STAGE_ARGS) {
    __shared__ double sH[kDetailStagedRows][32];
    __shared__ float2 sE[kDetailStagedRows][32];
    __shared__ float sD[kDetailRowsTall + 2][33];
    __shared__ float sX[kDetailRowsTall + 2][33];
    __shared__ DetailRows R;
    __shared__ FrameJob sJob;
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    stageJob(jobs, f, sJob);
    const FrameJob &J = sJob;
    const int tile = blockIdx.x - tileStart[f];
    const int w = J.sw, h = J.sh, cw = J.cw, ch = J.ch;
    const int rowsOut = J.detailRows, rowsIn = rowsOut + 2;
    const int tilesX = (w + kDetailTile - 1) / kDetailTile;
    const int x0 = (tile % tilesX) * kDetailTile, y0 = (tile / tilesX) * rowsOut;
    const int lx = threadIdx.x, tid = threadIdx.y * 32 + lx;
    if (J.detailReach > 0) {
        // skip tiles whose samples no active pixel's transfer reads
        const int reach = J.detailReach;
        const int xa = max(0, x0 - reach), xb = min(w - 1, x0 + kDetailTile - 1 + reach);
        const int ya = max(0, y0 - reach), yb = min(h - 1, y0 + rowsOut - 1 + reach);
        const int wa = xa >> 5, wb = xb >> 5, nw = wb - wa + 1;
        bool any = false;
        for (int i = tid; i < (yb - ya + 1) * nw; i += 256) {
            const int yy = ya + i / nw, wd = wa + i % nw;
            uint32_t m = __ldg(J.mask + (size_t)yy * J.maskWords + wd);
            if (wd == wa)
                m &= ~0u << (xa & 31);
            if (wd == wb && (xb & 31) != 31)
                m &= (1u << ((xb & 31) + 1)) - 1u;
            any |= m != 0;
        }
        if (!__syncthreads_or(any))
            return;
    }
    const int c = iclamp(x0 - 1 + lx, 0, w - 1);
    const AxisView &ax = J.sax, &ay = J.say;
    const int supY = ay.sup;
    for (int i = tid; i < rowsIn * supY; i += 256) {
        const int k = i / supY, j = i - k * supY;
        const int rk = iclamp(y0 - 1 + k, 0, h - 1);
        R.w[k][j] = __ldg(ay.wd + (size_t)rk * supY + j);
    }
    if (tid < rowsIn) {
        const int rk = iclamp(y0 - 1 + tid, 0, h - 1);
        R.r[tid] = rk;
        R.ty0[tid] = __ldg(ay.start + rk);
        R.act[tid] = activityBits(ay.am + (size_t)rk * supY, supY);
        R.wsum[tid] = __ldg(ay.wsum + rk);
        R.wabs[tid] = __ldg(ay.wabs + rk);
        R.pos[tid] = __ldg(ay.pos + rk);
    }
    const int syLo = iclamp(__ldg(ay.start + iclamp(y0 - 1, 0, h - 1)), 0, ch - 1);
    const int syHi = iclamp(__ldg(ay.start + iclamp(y0 + rowsOut, 0, h - 1)) + supY - 1, 0, ch - 1);
    const int nRows = syHi - syLo + 1;
    const float *dgl = J.aff + 8 * (size_t)cw * ch;
    {
        // horizontal entries of column c on the chroma rows the tile reads
        const int supX = ax.sup;
        const int tx0 = __ldg(ax.start + c);
        const uint32_t act = activityBits(ax.am + (size_t)c * supX, supX);
        double wx[8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
            wx[i] = i < supX ? __ldg(ax.wd + (size_t)c * supX + i) : 0.0;
        for (int r = threadIdx.y; r < nRows; r += blockDim.y) {
            const float *row = dgl + (size_t)(syLo + r) * cw;
            double hv;
            float2 e;
            if (J.sNoClampX)
                detailEntry<true>(row, cw, tx0, wx, act, hv, e);
            else
                detailEntry<false>(row, cw, tx0, wx, act, hv, e);
            sH[r][lx] = hv;
            sE[r][lx] = e;
        }
    }
    __syncthreads();
    {
        const float wsX = __ldg(ax.wsum + c), waX = __ldg(ax.wabs + c), posX = __ldg(ax.pos + c);
        for (int k = threadIdx.y; k < rowsIn; k += blockDim.y) {
            float mn, mx;
            double v = J.sNoClampY ? detailVertical<true>(R, sH, sE, k, lx, syLo, ch, mn, mx)
                                   : detailVertical<false>(R, sH, sE, k, lx, syLo, ch, mn, mx);
            const double ws = (double)wsX * (double)R.wsum[k];
            const double wa = (double)waX * (double)R.wabs[k];
            if (ws > 1e-6 && ws >= 0.05 * wa)
                v /= ws;
            else
                v = bilinearAt(dgl, cw, ch, posX, R.pos[k]);
            if (J.clampHull)
                v = sclamp(v, (double)(mn - J.margin), (double)(mx + J.margin));
            sD[k][lx] = ldf(J.Y + (size_t)R.r[k] * w + c) - (float)v;
        }
    }
    __syncthreads();
    const float (*src)[33] = sD;
    if (J.nyqX) {
        if (lx >= 1 && lx <= kDetailTile)
            for (int k = threadIdx.y; k < rowsIn; k += blockDim.y)
                sX[k][lx] = 0.25f * sD[k][lx - 1] + 0.5f * sD[k][lx] + 0.25f * sD[k][lx + 1];
        __syncthreads();
        src = sX;
    }
    const int x = x0 - 1 + lx;
    if (lx < 1 || lx > kDetailTile || x >= w)
        return;
    float *dst = const_cast<float *>(J.detailSrc);
    for (int k = 1 + threadIdx.y; k <= rowsOut; k += blockDim.y) {
        const int y = y0 - 1 + k;
        if (y >= h)
            break;
        const float val = J.nyqY ? 0.25f * src[k - 1][lx] + 0.5f * src[k][lx] + 0.25f * src[k + 1][lx]
                                 : src[k][lx];
        dst[(size_t)y * w + x] = val;
    }
}

// One dyadic pass: x passes (steps 1,2,4..) then y passes; ping-pong
// between detailTmp and detailTmp2.
__global__ void k_detail_nyq(LGCR_STAGE_ARGS, int pass) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int x, y;
    tile32x8(blockIdx.x - tileStart[f], J.sw, x, y);
    if (x >= J.sw || y >= J.sh)
        return;
    const float *src = (pass & 1) ? J.detailTmp2 : J.detailTmp;
    float *dst = (pass & 1) ? J.detailTmp : J.detailTmp2;
    const int w = J.sw, h = J.sh;
    float a, b, c;
    if (pass < J.nyqX) {
        const int step = 1 << pass;
        const float *row = src + (size_t)y * w;
        a = row[max(0, x - step)]; b = row[x]; c = row[min(w - 1, x + step)];
    } else {
        const int step = 1 << (pass - J.nyqX);
        a = src[(size_t)max(0, y - step) * w + x];
        b = src[(size_t)y * w + x];
        c = src[(size_t)min(h - 1, y + step) * w + x];
    }
    dst[(size_t)y * w + x] = 0.25f * a + 0.5f * b + 0.25f * c;
}

__global__ void k_detail_resize_h(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int x, y;
    tile32x8(blockIdx.x - tileStart[f], J.W, x, y);
    if (x >= J.W || y >= J.sh)
        return;
    const WeightView &t = J.lumaH;
    const int s = __ldg(t.start + x);
    const float *wp = t.w + (size_t)x * t.sup;
    const float *row = J.detailSrc + (size_t)y * J.sw;
    double acc = 0.0;
    for (int j = 0; j < t.sup; ++j)
        acc = fma((double)__ldg(wp + j), (double)row[iclamp(s + j, 0, J.sw - 1)], acc);
    J.lumaTmp[(size_t)y * J.W + x] = (float)acc;
}

__global__ void k_detail_resize_v(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int x, y;
    tile32x8(blockIdx.x - tileStart[f], J.W, x, y);
    if (x >= J.W || y >= J.H)
        return;
    const WeightView &t = J.lumaV;
    const int s = __ldg(t.start + y);
    const float *wp = t.w + (size_t)y * t.sup;
    double acc = 0.0;
    for (int j = 0; j < t.sup; ++j)
        acc = fma((double)__ldg(wp + j),
                  (double)J.lumaTmp[(size_t)iclamp(s + j, 0, J.sh - 1) * J.W + x], acc);
    J.detail[(size_t)y * J.W + x] = (float)acc;
}

__global__ void k_detail_resize_radial(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int ox, oy;
    tile32x8(blockIdx.x - tileStart[f], J.W, ox, oy);
    if (ox >= J.W || oy >= J.H)
        return;
    const double sx = (double)J.sw / J.W, sy = (double)J.sh / J.H;
    const double widen = fmax(1.0, fmax(sx, sy));
    const float invW = (float)(1.0 / widen);
    const int radius = (int)ceil(J.support * widen);
    const int sup = 2 * radius;
    const double cy = (oy + 0.5) * sy - 0.5;
    const int y0 = (int)ceil(cy - radius);
    const double cx = (ox + 0.5) * sx - 0.5;
    const int x0 = (int)ceil(cx - radius);
    double acc = 0.0, wsum = 0.0;
    for (int j = 0; j < sup; ++j) {
        const int ty = iclamp(y0 + j, 0, J.sh - 1);
        const float dy = (float)((y0 + j - cy) * invW);
        const float *row = J.detailSrc + (size_t)ty * J.sw;
        for (int i = 0; i < sup; ++i) {
            const int tx = iclamp(x0 + i, 0, J.sw - 1);
            const float dx = (float)((x0 + i - cx) * invW);
            const float w = lutLookupDev(J.lut, J.lutN, sqrtf(dx * dx + dy * dy) * J.lutScale);
            acc = fma((double)w, (double)row[tx], acc);
            wsum += (double)w;
        }
    }
    J.detail[(size_t)oy * J.W + ox] = (float)(wsum > 1e-6 ? acc / wsum : 0.0);
}

__device__ __forceinline__ bool activeOut(const FrameJob &J, int ox, int oy) {
    if (!J.sparse)
        return true;
    const int mx = J.sameSize ? ox : min(J.sw - 1, (int)((long long)ox * J.sw / J.W));
    const int my = J.sameSize ? oy : min(J.sh - 1, (int)((long long)oy * J.sh / J.H));
    return maskAt(J, mx, my) != 0;
}

// Detail transfer of one active output pixel (detailTransferImpl,
// src/algos.cpp:1587-1698).
__device__ __forceinline__ void transferPixel(const FrameJob &J, int ox, int oy) {
    const AxisView &ax = J.ax, &ay = J.ay;
    const int lxi = __ldg(ax.lbI0 + ox), lyi = __ldg(ay.lbI0 + oy);
    const float lxf = __ldg(ax.lbF + ox), lyf = __ldg(ay.lbF + oy);
    const float jxx = bilinearFast(J.jxx, J.sw, J.sh, lxi, lxf, lyi, lyf);
    const float jxy = bilinearFast(J.jxy, J.sw, J.sh, lxi, lxf, lyi, lyf);
    const float jyy = bilinearFast(J.jyy, J.sw, J.sh, lxi, lxf, lyi, lyf);
    const TensorDir dir = principalDirection(jxx, jxy, jyy);
    const int cxi = __ldg(ax.cbI0 + ox), cyi = __ldg(ay.cbI0 + oy);
    const float cxf = __ldg(ax.cbF + ox), cyf = __ldg(ay.cbF + oy);
    const int cw = J.cw, ch = J.ch;
    const size_t C = (size_t)cw * ch;
    // (aU, aV, g, rng) and (mnU, mxU, mnV, mxV), bilinear per component
    const float4 amap = bilinearFast4(reinterpret_cast<const float4 *>(J.aff), cw, ch, cxi, cxf, cyi, cyf);
    const float q = amap.z;
    float g = (1.0f - J.qgate * (1.0f - q)) * J.strength;
    if (J.useMs) {
        const float ms = bilinearFast(J.ms, cw, ch, cxi, cxf, cyi, cyf);
        g *= 1.0f - J.msStrength * (1.0f - ms);
    }
    const float au = amap.x;
    const float av = amap.y;
    const float coherence = dir.coherence;
    const float tx = -dir.ny, ty = dir.nx;
    const float *dl = J.detail;
    const float dc = dl[(size_t)oy * J.W + ox];
    const float s = 1.0f + J.stretch * coherence;
    const float dtp = bilinearAt(dl, J.W, J.H, (float)ox + tx * s, (float)oy + ty * s);
    const float dtm = bilinearAt(dl, J.W, J.H, (float)ox - tx * s, (float)oy - ty * s);
    const float dt = 0.25f * dtp + 0.5f * dc + 0.25f * dtm;
    const float det = dc + (dt - dc) * coherence;
    const float cap = 0.5f * amap.w;
    const float cu = sclamp(g * au * det, -cap, cap);
    const float cv = sclamp(g * av * det, -cap, cap);
    const size_t o = (size_t)oy * J.W + ox;
    const float ru = J.oU[o], rv = J.oV[o];
    float ou = ru + cu, ov = rv + cv;
    if (J.clampHull) {
        const float ar = J.margin;
        const float4 hull = bilinearFast4(reinterpret_cast<const float4 *>(J.aff + 4 * C), cw, ch, cxi,
                                          cxf, cyi, cyf);
        const float loU = smin(ru, hull.x - ar);
        const float hiU = smax(ru, hull.y + ar);
        const float loV = smin(rv, hull.z - ar);
        const float hiV = smax(rv, hull.w + ar);
        ou = sclamp(ou, loU, hiU);
        ov = sclamp(ov, loV, hiV);
    }
    if (J.finalInTransfer) {
        storeChroma(J, 1, ox, oy, ou);
        storeChroma(J, 2, ox, oy, ov);
    } else {
        J.oU[o] = ou;
        J.oV[o] = ov;
    }
}
__global__ void k_detail_transfer(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int ox, oy;
    tile32x8(blockIdx.x - tileStart[f], J.W, ox, oy);
    if (ox >= J.W || oy >= J.H || !activeOut(J, ox, oy))
        return;
    transferPixel(J, ox, oy);
}

// Sparse frames: a persistent grid walks the frames' compacted work lists of
// active output pixels (built by the workset stage), so no lane idles on an
// inactive pixel. Each block builds the prefix of the listed frames' list
// lengths in shared memory and strides over the concatenated work.
constexpr int kXferMaxFrames = 1024;

__global__ void __launch_bounds__(256)
k_detail_transfer_list(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    __shared__ unsigned long long pre[kXferMaxFrames + 1];
    for (int chunk = 0; chunk < njobs; chunk += kXferMaxFrames) {
        const int n = min(kXferMaxFrames, njobs - chunk);
        if (threadIdx.x == 0) {
            unsigned long long acc = 0;
            for (int i = 0; i < n; ++i) {
                pre[i] = acc;
                const FrameJob &J = jobs[chunk + i];
                if (J.xferListed)
                    acc += J.counters[kCntActiveOutput];
            }
            pre[n] = acc;
        }
        __syncthreads();
        const unsigned long long total = pre[n];
        for (unsigned long long w = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; w < total;
             w += (unsigned long long)gridDim.x * blockDim.x) {
            int lo = 0, hi = n - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (pre[mid] <= w) lo = mid; else hi = mid - 1;
            }
            const FrameJob &J = jobs[chunk + lo];
            const uint32_t pix = __ldg(J.actList + (w - pre[lo]));
            transferPixel(J, (int)(pix & 0xffffu), (int)(pix >> 16));
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// algo 4
// ---------------------------------------------------------------------------
__device__ __forceinline__ float pointLuma(const FrameJob &J, int x, int y) {
    return bilinearFast(J.Y, J.sw, J.sh, __ldg(J.lsX + x), __ldg(J.lsXf + x),
                        __ldg(J.lsY + y), __ldg(J.lsYf + y));
}

// LGF regression per chroma sample: 5x5 sums of {l, l^2, u, l*u, v, l*v}
// with l the point-sampled luma; conf = var/(var+eps) (x cedge fade), then
// the mutual-structure fade. Integer output: all samples; float: ROI only.
//
// A block stages its tile's point-sampled luma (computed once per sample,
// not once per window that covers it) and U, V with a 2-sample clamped halo
// in shared memory; each thread then sums its clipped 5x5 window from there
// in the same raster order, so the sums are the reference's. Tiles without
// an ROI sample only store the maps' zeros.
constexpr int kLgfTile = 1024;               // (bx + 4) * (by + 4) of every block shape used

__global__ void __launch_bounds__(256)
k_lgf(LGCR_STAGE_ARGS) {
    __shared__ float sL[kLgfTile], sU[kLgfTile], sV[kLgfTile];
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int w = J.cw, h = J.ch;
    const int bx = blockDim.x, by = blockDim.y;
    const int tile = blockIdx.x - tileStart[f];
    const int tilesX = (w + bx - 1) / bx;
    const int x0 = (tile % tilesX) * bx, y0 = (tile / tilesX) * by;
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    const bool inside = x < w && y < h;
    const size_t o = inside ? (size_t)y * w + x : 0;
    const bool work = inside && (!J.lgfRoiOnly || J.roi[o] != 0);
    const int lx = bx + 4, ly = by + 4;
    const bool staged = lx * ly <= kLgfTile;
    if (!__syncthreads_or(work)) {
        // outside the ROI the maps hold zeros (buildLGFMaps fills them before
        // the ROI pass, recon.cpp:1541-1548); the blend reads them wherever
        // w2 or w3 reaches 1e-4, which includes samples outside the ROI
        if (inside) {
            const size_t C = (size_t)w * h;
#pragma unroll
            for (int k = 0; k < 6; ++k)
                J.lgf[k * C + o] = 0.0f;
        }
        return;
    }
    if (staged) {
        for (int k = threadIdx.y * bx + threadIdx.x; k < lx * ly; k += bx * by) {
            const int px = iclamp(x0 - 2 + k % lx, 0, w - 1), py = iclamp(y0 - 2 + k / lx, 0, h - 1);
            sL[k] = pointLuma(J, px, py);
            sU[k] = ldf(J.U + (size_t)py * w + px);
            sV[k] = ldf(J.V + (size_t)py * w + px);
        }
    }
    __syncthreads();
    if (!inside)
        return;
    if (!work) {
        const size_t C = (size_t)w * h;
#pragma unroll
        for (int k = 0; k < 6; ++k)
            J.lgf[k * C + o] = 0.0f;
        return;
    }
    const int top = max(0, y - 2), bottom = min(h - 1, y + 2);
    const int left = max(0, x - 2), right = min(w - 1, x + 2);
    double s[6] = {0, 0, 0, 0, 0, 0};
    if (staged) {
        for (int py = top; py <= bottom; ++py) {
            const int r = (py - y0 + 2) * lx - x0 + 2;
            for (int px = left; px <= right; ++px) {
                const double lv = sL[r + px];
                const double u = sU[r + px], v = sV[r + px];
                s[0] += lv; s[1] += lv * lv; s[2] += u; s[3] += lv * u; s[4] += v; s[5] += lv * v;
            }
        }
    } else {
        for (int py = top; py <= bottom; ++py)
            for (int px = left; px <= right; ++px) {
                const double lv = pointLuma(J, px, py);
                const double u = ldf(J.U + (size_t)py * w + px), v = ldf(J.V + (size_t)py * w + px);
                s[0] += lv; s[1] += lv * lv; s[2] += u; s[3] += lv * u; s[4] += v; s[5] += lv * v;
            }
    }
    const int n = (right - left + 1) * (bottom - top + 1);
    const double eps = J.lgfEps;
    const double meanY = s[0] / n;
    const double var = s[1] / n - meanY * meanY;
    const double meanU = s[2] / n, meanV = s[4] / n;
    const double slopeU = (s[3] / n - meanY * meanU) / (var + eps);
    const double slopeV = (s[5] / n - meanY * meanV) / (var + eps);
    const size_t C = (size_t)w * h;
    float *L = J.lgf;
    L[0 * C + o] = (float)slopeU;
    L[1 * C + o] = (float)(meanU - slopeU * meanY);
    L[3 * C + o] = (float)slopeV;
    L[4 * C + o] = (float)(meanV - slopeV * meanY);
    const float base = (float)(var / (var + eps));
    float confU = base, confV = base;
    if (J.cedge) {
        auto lsAt = [&](int xx, int yy) { return pointLuma(J, iclamp(xx, 0, w - 1), iclamp(yy, 0, h - 1)); };
        const float lgx = (lsAt(x + 1, y) - lsAt(x - 1, y)) * 0.5f;
        const float lgy = (lsAt(x, y + 1) - lsAt(x, y - 1)) * 0.5f;
        const float gl = hypotf(lgx, lgy);
        auto fade = [&](const float *P) {
            float mn = P[(size_t)max(0, y - 2) * w + max(0, x - 2)], mx = mn;
            for (int py = y - 2; py <= y + 2; ++py)
                for (int px = x - 2; px <= x + 2; ++px) {
                    const float v = P[(size_t)iclamp(py, 0, h - 1) * w + iclamp(px, 0, w - 1)];
                    mn = smin(mn, v); mx = smax(mx, v);
                }
            const float range = mx - mn;
            if (gl <= 1e-9f || range <= 1e-6f)
                return 1.0f;
            auto at = [&](int xx, int yy) { return P[(size_t)iclamp(yy, 0, h - 1) * w + iclamp(xx, 0, w - 1)]; };
            const float cgx = (at(x + 1, y) - at(x - 1, y)) * 0.5f;
            const float cgy = (at(x, y + 1) - at(x, y - 1)) * 0.5f;
            const float gradN = fabsf(cgx * lgx / gl + cgy * lgy / gl);
            const float width = range / (gradN + 1e-6f);
            return sclamp((2.2f - width) / 0.7f, 0.0f, 1.0f);
        };
        confU *= fade(J.U);
        confV *= fade(J.V);
    }
    if (J.useMs) {
        const float fm = 1.0f - J.msStrength * (1.0f - J.ms[o]);
        confU *= fm;
        confV *= fm;
    }
    L[2 * C + o] = confU;
    L[5 * C + o] = confV;
}

// Mark the 2x2 chroma footprint of output samples whose diagonal routing
// weight reaches 1e-4.
__global__ void k_roi(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int ox, oy;
    tile32x8(blockIdx.x - tileStart[f], J.W, ox, oy);
    if (ox >= J.W || oy >= J.H || !activeOut(J, ox, oy))
        return;
    if (J.selW3[(size_t)oy * J.W + ox] < 1e-4f)
        return;
    const int cx0 = __ldg(J.ax.cbI0 + ox), cx1 = min(cx0 + 1, J.cw - 1);
    const int cy0 = __ldg(J.ay.cbI0 + oy), cy1 = min(cy0 + 1, J.ch - 1);
    J.roi[(size_t)cy0 * J.cw + cx0] = 1;
    J.roi[(size_t)cy0 * J.cw + cx1] = 1;
    J.roi[(size_t)cy1 * J.cw + cx0] = 1;
    J.roi[(size_t)cy1 * J.cw + cx1] = 1;
}

__global__ void k_blend(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int ox, oy;
    tile32x8(blockIdx.x - tileStart[f], J.W, ox, oy);
    if (ox >= J.W || oy >= J.H)
        return;
    const size_t o = (size_t)oy * J.W + ox;
    // final sample: to the typed output when nothing follows the blend
    auto finish = [&](float u, float v) {
        if (J.blendStores) {
            storeChroma(J, 1, ox, oy, u);
            storeChroma(J, 2, ox, oy, v);
        } else {
            J.oU[o] = u;
            J.oV[o] = v;
        }
    };
    if (!activeOut(J, ox, oy)) {
        if (J.blendStores)
            finish(J.oU[o], J.oV[o]);
        return;
    }
    const float lam = J.strength4;
    const bool compressed = J.sparse &&
        (unsigned long long)J.counters[kCntActiveOutput] * 2ull < (unsigned long long)J.W * J.H;
    const int cw = J.cw, ch = J.ch;
    const size_t C = (size_t)cw * ch;
    const int cx = __ldg(J.ax.cbI0 + ox), cy = __ldg(J.ay.cbI0 + oy);
    const float cxf = __ldg(J.ax.cbF + ox), cyf = __ldg(J.ay.cbF + oy);
    const float plainU = J.oU[o], plainV = J.oV[o];
    if (compressed) {
        const float w3 = lam * J.selW3[o];
        float valueU = plainU + lam * J.gU[o];
        float valueV = plainV + lam * J.gV[o];
        if (w3 != 0.0f) {
            const float luma = bilinearFast(J.Y, J.sw, J.sh, __ldg(J.ax.lbI0 + ox), __ldg(J.ax.lbF + ox),
                                            __ldg(J.ay.lbI0 + oy), __ldg(J.ay.lbF + oy));
            const float au = bilinearFast(J.lgf + 0 * C, cw, ch, cx, cxf, cy, cyf);
            const float bu = bilinearFast(J.lgf + 1 * C, cw, ch, cx, cxf, cy, cyf);
            const float cu = bilinearFast(J.lgf + 2 * C, cw, ch, cx, cxf, cy, cyf);
            const float av = bilinearFast(J.lgf + 3 * C, cw, ch, cx, cxf, cy, cyf);
            const float bv = bilinearFast(J.lgf + 4 * C, cw, ch, cx, cxf, cy, cyf);
            const float cv = bilinearFast(J.lgf + 5 * C, cw, ch, cx, cxf, cy, cyf);
            valueU += w3 * cu * (au * luma + bu - plainU);
            valueV += w3 * cv * (av * luma + bv - plainV);
        }
        finish(valueU, valueV);
        return;
    }
    const float w2v = J.selW2[o] * lam;
    const float w3v = J.selW3[o] * lam;
    if (w2v < 1e-4f && w3v < 1e-4f) {
        if (J.blendStores)
            finish(plainU, plainV);
        return;
    }
    const float L0 = bilinearFast(J.Y, J.sw, J.sh, __ldg(J.ax.lbI0 + ox), __ldg(J.ax.lbF + ox),
                                  __ldg(J.ay.lbI0 + oy), __ldg(J.ay.lbF + oy));
    const float au = bilinearFast(J.lgf + 0 * C, cw, ch, cx, cxf, cy, cyf);
    const float bu = bilinearFast(J.lgf + 1 * C, cw, ch, cx, cxf, cy, cyf);
    const float cu = bilinearFast(J.lgf + 2 * C, cw, ch, cx, cxf, cy, cyf);
    const float av = bilinearFast(J.lgf + 3 * C, cw, ch, cx, cxf, cy, cyf);
    const float bv = bilinearFast(J.lgf + 4 * C, cw, ch, cx, cxf, cy, cyf);
    const float cv = bilinearFast(J.lgf + 5 * C, cw, ch, cx, cxf, cy, cyf);
    finish(plainU + (w2v * (J.gU[o] - plainU) + w3v * cu * (au * L0 + bu - plainU)),
           plainV + (w2v * (J.gV[o] - plainV) + w3v * cv * (av * L0 + bv - plainV)));
}

} // namespace lgcr_b200
