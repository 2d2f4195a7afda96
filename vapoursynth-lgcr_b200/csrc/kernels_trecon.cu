// TRecon preparation kernels:
//   k_trecon_convert  planeToFloat of the frame and its neighbours
//                     (tReconGetFrame's extract, src/plugin.cpp:771-790)
//   k_trecon_lc       the neighbours' footprint luma maps (buildLcMap,
//                     src/maps.cpp:425-499)
//   k_block_match     blockMatch, src/algos.cpp:683-755
//   k_chroma_consist  applyChromaConsistency, src/algos.cpp:757-807
//
// Block matching: one CTA per (16x16 block, neighbour). The block's
// subsampled luma (every second row and column) sits in shared memory; each
// thread takes candidate displacements in scan order and sums |cur - nbr| in
// the reference's sample order, so every candidate's SAD is the reference's
// float. The sequential choice (strictly smaller SAD, or equal SAD with a
// smaller |dx|+|dy|) selects the lexicographic minimum of (SAD, |dx|+|dy|,
// scan index): a 64-bit key (SAD bits, norm, index) reduced with min.
//
// Consistency: one CTA per (block, neighbour); the block's chroma deltas are
// sorted in shared memory (bitonic, padded with +inf) for the median.
#include "trecon.h"

#include <algorithm>

namespace lgcr_b200 {

namespace {

template <int KIND>
__device__ __forceinline__ float rawFloat(const void *base, long long pitch, int x, int y,
                                          double scale, double off) {
    const char *row = static_cast<const char *>(base) + (long long)y * pitch;
    if (KIND == kU8)
        return (float)((double)__ldg(reinterpret_cast<const unsigned char *>(row) + x) * scale + off);
    if (KIND == kU16)
        return (float)((double)__ldg(reinterpret_cast<const unsigned short *>(row) + x) * scale + off);
    return __ldg(reinterpret_cast<const float *>(row) + x) + 0.0f;   // s * 1.0 + 0.0
}

// blockIdx.y: frame * 3 + plane
template <int KIND>
__global__ void __launch_bounds__(256) k_trecon_convert(const TReconPrep P) {
    const int frame = blockIdx.y / 3, plane = blockIdx.y % 3;
    const int w = plane ? P.cw : P.sw, h = plane ? P.ch : P.sh;
    const double off = plane ? P.cOffset : 0.0;
    float *dst = P.f[frame][plane];
    const size_t n = (size_t)w * h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / w), x = (int)(i % w);
        dst[i] = rawFloat<KIND>(P.in[frame][plane], P.inPitch[frame][plane], x, y, P.yScale, off);
    }
}

// blockIdx.y: neighbour - 1
__global__ void __launch_bounds__(256) k_trecon_lc(const TReconPrep P) {
    const int k = 1 + blockIdx.y;
    const float *Y = P.f[k][0];
    float *lc = P.lc[k];
    const size_t n = (size_t)P.cw * P.ch;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int cy = (int)(i / P.cw), cx = (int)(i % P.cw);
        const int xb = __ldg(P.lcXb + cx), xe = __ldg(P.lcXe + cx);
        const int yb = __ldg(P.lcYb + cy), ye = __ldg(P.lcYe + cy);
        double sum = 0.0;
        for (int j = yb; j < ye; ++j)
            for (int x = xb; x < xe; ++x)
                sum += (double)ldf(Y + (size_t)j * P.sw + x);
        lc[i] = (float)(sum / ((double)(xe - xb) * (double)(ye - yb)));
    }
}

constexpr int kMatchThreads = 256;

// blockIdx.x: block index, blockIdx.y: neighbour - 1
__global__ void __launch_bounds__(kMatchThreads) k_block_match(const TReconPrep P) {
    __shared__ float cur[kTReconBlock / 2][kTReconBlock / 2];
    __shared__ unsigned long long best[kMatchThreads / 32];
    __shared__ float sad0Shared;
    const int k = 1 + blockIdx.y;
    const int bx = blockIdx.x % P.bw, by = blockIdx.x / P.bw;
    const int w = P.sw, h = P.sh;
    const int x0 = bx * kTReconBlock, y0 = by * kTReconBlock;
    const int bw_ = min(kTReconBlock, w - x0), bh_ = min(kTReconBlock, h - y0);
    const int ni = (bw_ + 1) / 2, nj = (bh_ + 1) / 2;
    const float *C = P.f[0][0], *N = P.f[k][0];
    for (int t = threadIdx.x; t < ni * nj; t += blockDim.x) {
        const int i = t % ni, j = t / ni;
        cur[j][i] = ldf(C + (size_t)(y0 + 2 * j) * w + x0 + 2 * i);
    }
    __syncthreads();
    const int s = P.search, side = 2 * s + 1, cands = side * side;
    unsigned long long key = ~0ull;
    for (int c = threadIdx.x; c < cands; c += blockDim.x) {
        const int dy = c / side - s, dx = c % side - s;
        if (x0 + dx < 0 || y0 + dy < 0 || x0 + dx + bw_ > w || y0 + dy + bh_ > h)
            continue;
        const float *nb = N + (size_t)(y0 + dy) * w + x0 + dx;
        float sad = 0.0f;
        for (int j = 0; j < nj; ++j) {
            const float *row = nb + (size_t)(2 * j) * w;
            for (int i = 0; i < ni; ++i)
                sad += fabsf(cur[j][i] - ldf(row + 2 * i));
        }
        if (dx == 0 && dy == 0)
            sad0Shared = sad;
        const unsigned norm = (unsigned)(abs(dx) + abs(dy));
        const unsigned long long kk = ((unsigned long long)__float_as_uint(sad) << 32) |
                                      ((unsigned long long)norm << 16) | (unsigned long long)c;
        key = kk < key ? kk : key;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_down_sync(0xffffffffu, key, o);
        key = other < key ? other : key;
    }
    if ((threadIdx.x & 31) == 0)
        best[threadIdx.x >> 5] = key;
    __syncthreads();
    if (threadIdx.x != 0)
        return;
    for (int q = 1; q < kMatchThreads / 32; ++q)
        key = best[q] < key ? best[q] : key;
    const int c = (int)(key & 0xffffu);
    int bdy = c / side - s, bdx = c % side - s;
    float bestSad = __uint_as_float((unsigned)(key >> 32));
    const float sad0 = sad0Shared;
    // subsampled block statistics in the reference's order
    double sum = 0.0, sum2 = 0.0;
    for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i) {
            const float v = cur[j][i];
            sum += v;
            sum2 += (double)v * v;
        }
    const float npix = (float)(ni * nj);
    // zero-motion snap
    if ((bdx != 0 || bdy != 0) && sad0 - bestSad <= 0.10f * P.tsad * npix) {
        bdx = 0;
        bdy = 0;
        bestSad = sad0;
    }
    const size_t idx = (size_t)by * P.bw + bx;
    P.mvx[k][idx] = (short)bdx;
    P.mvy[k][idx] = (short)bdy;
    const float sadPx = bestSad / npix;
    const double m = sum / npix;
    const double vr = sum2 / npix - m * m;
    const float var = (float)(0.0 < vr ? vr : 0.0);
    const float invT2 = 1.0f / (P.tsad * P.tsad);
    const float matchQ = 1.0f / (1.0f + sadPx * sadPx * invT2);
    const float uniq = var / (var + 0.25f * P.tsad * P.tsad);
    P.conf[k][idx] = matchQ * uniq;
}

constexpr int kConsistMax = 256;            // 16 x 16 deltas at most (4:4:4)

__global__ void __launch_bounds__(kConsistMax) k_chroma_consist(const TReconPrep P) {
    __shared__ float d[kConsistMax];
    const int k = 1 + blockIdx.y;
    const int bx = blockIdx.x % P.bw, by = blockIdx.x / P.bw;
    const size_t bi = (size_t)by * P.bw + bx;
    const float conf = P.conf[k][bi];
    if (conf <= 0.0f)
        return;                                      // uniform over the block
    const int cw = P.cw, ch = P.ch;
    const int lx0 = bx * kTReconBlock, ly0 = by * kTReconBlock;
    const int lx1 = min(P.sw, lx0 + kTReconBlock), ly1 = min(P.sh, ly0 + kTReconBlock);
    const int cx0 = iclamp((int)floor(lx0 / P.rw), 0, cw - 1);
    const int cy0 = iclamp((int)floor(ly0 / P.rh), 0, ch - 1);
    const int cx1 = iclamp((int)ceil(lx1 / P.rw), cx0 + 1, cw);
    const int cy1 = iclamp((int)ceil(ly1 / P.rh), cy0 + 1, ch);
    const double mx = P.mvx[k][bi] / P.rw, my = P.mvy[k][bi] / P.rh;
    const int nx = cx1 - cx0, n = nx * (cy1 - cy0);
    if (n > kConsistMax)
        return;                                      // not reachable: TRecon ratios are 1..2
    const float *cu = P.f[0][1], *cv = P.f[0][2], *nu = P.f[k][1], *nv = P.f[k][2];
    for (int t = threadIdx.x; t < kConsistMax; t += blockDim.x) {
        float v = __int_as_float(0x7f800000);        // +inf pads the sort
        if (t < n) {
            const int cx = cx0 + t % nx, cy = cy0 + t / nx;
            const int tx = iclamp((int)llround(cx + mx), 0, cw - 1);
            const int ty = iclamp((int)llround(cy + my), 0, ch - 1);
            const size_t o = (size_t)cy * cw + cx, q = (size_t)ty * cw + tx;
            v = smax(fabsf(ldf(cu + o) - ldf(nu + q)), fabsf(ldf(cv + o) - ldf(nv + q)));
        }
        d[t] = v;
    }
    __syncthreads();
    // bitonic sort of the padded deltas (ascending)
    for (int size = 2; size <= kConsistMax; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const int t = threadIdx.x;
            const int partner = t ^ stride;
            if (partner > t) {
                const bool up = (t & size) == 0;
                const float a = d[t], b = d[partner];
                if ((a > b) == up) {
                    d[t] = b;
                    d[partner] = a;
                }
            }
            __syncthreads();
        }
    if (threadIdx.x != 0)
        return;
    const int mid = n / 2;
    float median = d[mid];
    if ((n & 1) == 0)
        median = 0.5f * (d[mid - 1] + median);
    const float ratio = median / 0.04f;
    const float ratio2 = ratio * ratio;
    const float cconf = 1.0f / (1.0f + ratio2 * ratio2);
    P.conf[k][bi] = conf * cconf;
}

template <int KIND>
void convertKind(const TReconPrep &P, cudaStream_t s) {
    const size_t most = (size_t)P.sw * P.sh;
    const int blocks = (int)std::min<size_t>((most + 255) / 256, 1184);
    k_trecon_convert<KIND><<<dim3(blocks, 3 * P.frames), 256, 0, s>>>(P);
}

} // namespace

int launchTReconPrep(const TReconPrep &P, cudaStream_t s) {
    const int nbrs = P.frames - 1;
    if (nbrs <= 0)
        return 0;
    switch (P.kind) {
    case kU8: convertKind<kU8>(P, s); break;
    case kU16: convertKind<kU16>(P, s); break;
    default: convertKind<kF32>(P, s); break;
    }
    const size_t cn = (size_t)P.cw * P.ch;
    k_trecon_lc<<<dim3((int)std::min<size_t>((cn + 255) / 256, 1184), nbrs), 256, 0, s>>>(P);
    k_block_match<<<dim3(P.bw * P.bh, nbrs), kMatchThreads, 0, s>>>(P);
    k_chroma_consist<<<dim3(P.bw * P.bh, nbrs), kConsistMax, 0, s>>>(P);
    return cudaGetLastError() == cudaSuccess ? 4 : -1;
}

} // namespace lgcr_b200
