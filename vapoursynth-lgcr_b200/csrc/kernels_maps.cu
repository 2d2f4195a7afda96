// Map-building stages of the Recon path (all HBM-bound stencils):
//   k_convert      planeToFloat                       src/lgcr.h:986-995
//   k_tensor       sobelTensor3x3 + trust seed        src/maps.cpp:9-168
//   k_lc           buildLcMap (scalar footprint sum)  src/maps.cpp:425-499
//   k_dilate_h/v   buildTrustMask dilation            src/maps.cpp:280-340
//   k_mark_chroma  buildSparseWorkset chroma mask     src/maps.cpp:342-422
//   k_gate         buildMutualGate                    src/maps.cpp:831-948
#include "kernels.cuh"

namespace lgcr_b200 {

// ---------------------------------------------------------------------------
// input conversion: one thread per luma pixel (also converts the chroma
// sample at the same coordinates when it exists) and, for same-size output,
// copies the luma code to the output plane (the shared luma plane).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float loadSample(const FrameJob &J, int plane, int x, int y) {
    const char *row = static_cast<const char *>(J.in[plane]) + (long long)y * J.inPitch[plane];
    if (J.inKind == kF32)
        return reinterpret_cast<const float *>(row)[x];
    const double s = (J.inKind == kU8) ? (double)reinterpret_cast<const uint8_t *>(row)[x]
                                       : (double)reinterpret_cast<const uint16_t *>(row)[x];
    const double off = plane == 0 ? 0.0 : J.cOffset;
    return (float)(s * J.yScale + off);
}

__global__ void k_convert(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart,
                          int njobs) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int tilesX = (J.sw + 31) / 32;
    const int x = (tile % tilesX) * 32 + threadIdx.x;
    const int y = (tile / tilesX) * 8 + threadIdx.y;
    if (x >= J.sw || y >= J.sh)
        return;
    if (x == 0 && y == 0)
        for (int k = 0; k < kCntCount; ++k)
            J.counters[k] = 0ull;
    if (J.Yw)
        J.Yw[(size_t)y * J.sw + x] = loadSample(J, 0, x, y);
    if (J.writeLuma && J.sameSize) {
        const char *src = static_cast<const char *>(J.in[0]) + (long long)y * J.inPitch[0];
        char *dst = static_cast<char *>(J.out[0]) + (long long)y * J.outPitch[0];
        if (J.inKind == kU8) reinterpret_cast<uint8_t *>(dst)[x] = reinterpret_cast<const uint8_t *>(src)[x];
        else if (J.inKind == kU16) reinterpret_cast<uint16_t *>(dst)[x] = reinterpret_cast<const uint16_t *>(src)[x];
        else reinterpret_cast<float *>(dst)[x] = reinterpret_cast<const float *>(src)[x];
    }
    if (x < J.cw && y < J.ch) {
        const size_t o = (size_t)y * J.cw + x;
        if (J.cmask) J.cmask[o] = 0;
        if (J.roi) J.roi[o] = 0;
        const float u = loadSample(J, 1, x, y), v = loadSample(J, 2, x, y);
        if (J.Uw) J.Uw[o] = u;
        if (J.Vw) J.Vw[o] = v;
        if (J.uvd) reinterpret_cast<double2 *>(J.uvd)[o] = make_double2((double)u, (double)v);
    }
}

// ---------------------------------------------------------------------------
// Structure tensor: Sobel/8 gradients (clamped), vertical 3-row sums of the
// outer products, horizontal 3-tap box with the reference's border rule
// ((2a+b)/9 and (a+2b)/9 at the ends, *(1/9) inside), trust seed
// jxx + jyy > thr.  Tile TX x TY with a 2-pixel clamped halo in shared.
// ---------------------------------------------------------------------------
constexpr int TT_X = 32, TT_Y = 16;

__global__ void __launch_bounds__(TT_X * 8)
k_tensor(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    __shared__ float ys[TT_Y + 4][TT_X + 4];
    __shared__ float gxs[TT_Y + 2][TT_X + 2];
    __shared__ float gys[TT_Y + 2][TT_X + 2];
    __shared__ float vxx[TT_Y][TT_X + 2], vxy[TT_Y][TT_X + 2], vyy[TT_Y][TT_X + 2];
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int w = J.sw, h = J.sh;
    const int tilesX = (w + TT_X - 1) / TT_X;
    const int x0 = (tile % tilesX) * TT_X, y0 = (tile / tilesX) * TT_Y;
    const int tid = threadIdx.y * TT_X + threadIdx.x;
    const int nthreads = TT_X * 8;
    const float *Y = J.Y;
    for (int i = tid; i < (TT_Y + 4) * (TT_X + 4); i += nthreads) {
        const int r = i / (TT_X + 4), c = i % (TT_X + 4);
        const int gy = iclamp(y0 - 2 + r, 0, h - 1), gx = iclamp(x0 - 2 + c, 0, w - 1);
        ys[r][c] = ldf(Y + (size_t)gy * w + gx);
    }
    __syncthreads();
    // gradients at clamped positions of rows y0-1..y0+TY, cols x0-1..x0+TX
    for (int i = tid; i < (TT_Y + 2) * (TT_X + 2); i += nthreads) {
        const int r = i / (TT_X + 2), c = i % (TT_X + 2);
        const int gy = iclamp(y0 - 1 + r, 0, h - 1), gx = iclamp(x0 - 1 + c, 0, w - 1);
        const int sr = gy - y0 + 2, sc = gx - x0 + 2;
        const float tl = ys[sr - 1][sc - 1], t = ys[sr - 1][sc], tr = ys[sr - 1][sc + 1];
        const float l = ys[sr][sc - 1], rr = ys[sr][sc + 1];
        const float bl = ys[sr + 1][sc - 1], b = ys[sr + 1][sc], br = ys[sr + 1][sc + 1];
        gxs[r][c] = (tr + 2.0f * rr + br - tl - 2.0f * l - bl) * 0.125f;
        gys[r][c] = (bl + 2.0f * b + br - tl - 2.0f * t - tr) * 0.125f;
    }
    __syncthreads();
    // vertical sums for rows y0..y0+TY-1 at cols x0-1..x0+TX
    for (int i = tid; i < TT_Y * (TT_X + 2); i += nthreads) {
        const int r = i / (TT_X + 2), c = i % (TT_X + 2);
        const float ax0 = gxs[r][c], ax1 = gxs[r + 1][c], ax2 = gxs[r + 2][c];
        const float ay0 = gys[r][c], ay1 = gys[r + 1][c], ay2 = gys[r + 2][c];
        vxx[r][c] = ax0 * ax0 + ax1 * ax1 + ax2 * ax2;
        vxy[r][c] = ax0 * ay0 + ax1 * ay1 + ax2 * ay2;
        vyy[r][c] = ay0 * ay0 + ay1 * ay1 + ay2 * ay2;
    }
    __syncthreads();
    const float ninth = 1.0f / 9.0f;
    for (int i = tid; i < TT_Y * TT_X; i += nthreads) {
        const int r = i / TT_X, c = i % TT_X;
        const int x = x0 + c, y = y0 + r;
        if (x >= w || y >= h)
            continue;
        const int cc = c + 1;
        float oxx, oxy, oyy;
        if (x == 0) {
            const int rc = (w > 1) ? cc + 1 : cc;
            oxx = (2.0f * vxx[r][cc] + vxx[r][rc]) / 9.0f;
            oxy = (2.0f * vxy[r][cc] + vxy[r][rc]) / 9.0f;
            oyy = (2.0f * vyy[r][cc] + vyy[r][rc]) / 9.0f;
        } else if (x == w - 1) {
            oxx = (vxx[r][cc - 1] + 2.0f * vxx[r][cc]) / 9.0f;
            oxy = (vxy[r][cc - 1] + 2.0f * vxy[r][cc]) / 9.0f;
            oyy = (vyy[r][cc - 1] + 2.0f * vyy[r][cc]) / 9.0f;
        } else {
            oxx = ninth * (vxx[r][cc - 1] + vxx[r][cc] + vxx[r][cc + 1]);
            oxy = ninth * (vxy[r][cc - 1] + vxy[r][cc] + vxy[r][cc + 1]);
            oyy = ninth * (vyy[r][cc - 1] + vyy[r][cc] + vyy[r][cc + 1]);
        }
        const size_t o = (size_t)y * w + x;
        J.jxx[o] = oxx;
        J.jxy[o] = oxy;
        J.jyy[o] = oyy;
        if (J.trustOn)
            J.seed[o] = (oxx + oyy > J.trustThr) ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// Footprint luma per chroma sample: double sum in raster order.
// ---------------------------------------------------------------------------
__global__ void k_lc(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart,
                     int njobs) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int tilesX = (J.cw + 31) / 32;
    const int cx = (tile % tilesX) * 32 + threadIdx.x;
    const int cy = (tile / tilesX) * 8 + threadIdx.y;
    if (cx >= J.cw || cy >= J.ch)
        return;
    const int xb = __ldg(J.lcXb + cx), xe = __ldg(J.lcXe + cx);
    const int yb = __ldg(J.lcYb + cy), ye = __ldg(J.lcYe + cy);
    double sum = 0.0;
    for (int j = yb; j < ye; ++j) {
        const float *row = J.Y + (size_t)j * J.sw;
        for (int i = xb; i < xe; ++i)
            sum += (double)ldf(row + i);
    }
    J.lc[(size_t)cy * J.cw + cx] = (float)(sum / ((double)(xe - xb) * (double)(ye - yb)));
}

// ---------------------------------------------------------------------------
// Trust-mask dilation: square window of radius r (rolling population count in
// the reference; any-set in [x-r, x+r] here, same set).
// Horizontal: one block per (1024-pixel segment, row) with a shared prefix.
// ---------------------------------------------------------------------------
constexpr int DIL_SEG = 1024;
constexpr int DIL_MAXR = 512;

__global__ void __launch_bounds__(256)
k_dilate_h(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    __shared__ int pre[DIL_SEG + 2 * DIL_MAXR + 1];
    __shared__ int warpTot[8];
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int w = J.sw;
    const int segs = (w + DIL_SEG - 1) / DIL_SEG;
    const int y = tile / segs;
    const int x0 = (tile % segs) * DIL_SEG;
    const int r = J.dil;
    const int lo = x0 - r;
    const int span = DIL_SEG + 2 * r;         // prefix over [lo, lo+span)
    const uint8_t *src = J.seed + (size_t)y * w;
    // chunked block scan
    int carry = 0;
    for (int base = 0; base < span; base += 256) {
        const int i = base + threadIdx.x;
        const int gx = lo + i;
        int v = (i < span && gx >= 0 && gx < w) ? (src[gx] != 0) : 0;
        // warp inclusive scan
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            const int n = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += n;
        }
        if (lane == 31) warpTot[wid] = v;
        __syncthreads();
        int add = carry;
        for (int k = 0; k < wid; ++k) add += warpTot[k];
        if (i < span) pre[i + 1] = v + add;
        int total = 0;
        for (int k = 0; k < 8; ++k) total += warpTot[k];
        __syncthreads();
        carry += total;
    }
    if (threadIdx.x == 0) pre[0] = 0;
    __syncthreads();
    uint8_t *dst = J.mtmp + (size_t)y * w;
    for (int c = threadIdx.x; c < DIL_SEG; c += 256) {
        const int x = x0 + c;
        if (x >= w)
            break;
        // window [x-r, x+r] -> prefix indices [c, c+2r+1)
        dst[x] = (pre[c + 2 * r + 1] - pre[c]) != 0;
    }
}

// Vertical: 32 columns x DV_ROWS rows per block, rolling count per column
// over the tile rows (plus halo) staged in shared memory.
constexpr int DV_ROWS = 128;

__global__ void __launch_bounds__(32)
k_dilate_v(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    extern __shared__ uint8_t col[];   // (DV_ROWS + 2r) x 32
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int w = J.sw, h = J.sh, r = J.dil;
    const int tilesX = (w + 31) / 32;
    const int x = (tile % tilesX) * 32 + threadIdx.x;
    const int y0 = (tile / tilesX) * DV_ROWS;
    const int rows = DV_ROWS + 2 * r;
    for (int i = 0; i < rows; ++i) {
        const int gy = y0 - r + i;
        col[i * 32 + threadIdx.x] = (x < w && gy >= 0 && gy < h) ? J.mtmp[(size_t)gy * w + x] : 0;
    }
    __syncwarp();
    if (x >= w)
        return;
    int count = 0;
    for (int i = 0; i < 2 * r; ++i)
        count += col[i * 32 + threadIdx.x] != 0;
    for (int yy = 0; yy < DV_ROWS; ++yy) {
        const int y = y0 + yy;
        if (y >= h)
            break;
        count += col[(yy + 2 * r) * 32 + threadIdx.x] != 0;    // window [y-r, y+r]
        J.mask[(size_t)y * w + x] = count != 0;
        count -= col[yy * 32 + threadIdx.x] != 0;
    }
}

// ---------------------------------------------------------------------------
// Sparse workset: an output pixel is active when the mask sample its
// position maps to is set; active pixels mark the 2x2 chroma bilinear
// footprint. Counts active output pixels.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool outputActive(const FrameJob &J, int ox, int oy) {
    const int mx = J.sameSize ? ox : min(J.sw - 1, (int)((long long)ox * J.sw / J.W));
    const int my = J.sameSize ? oy : min(J.sh - 1, (int)((long long)oy * J.sh / J.H));
    return J.mask[(size_t)my * J.sw + mx] != 0;
}

__global__ void k_mark_chroma(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart,
                              int njobs) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int tilesX = (J.W + 31) / 32;
    const int ox = (tile % tilesX) * 32 + threadIdx.x;
    const int oy = (tile / tilesX) * 8 + threadIdx.y;
    bool active = false;
    if (ox < J.W && oy < J.H) {
        active = J.sparse ? outputActive(J, ox, oy) : true;
        if (active && J.sparse) {
            const int cx0 = __ldg(J.ax.cbI0 + ox);
            const int cx1 = min(cx0 + 1, J.cw - 1);
            const int cy0 = __ldg(J.ay.cbI0 + oy);
            const int cy1 = min(cy0 + 1, J.ch - 1);
            uint8_t *m = J.cmask;
            m[(size_t)cy0 * J.cw + cx0] = 1;
            m[(size_t)cy0 * J.cw + cx1] = 1;
            m[(size_t)cy1 * J.cw + cx0] = 1;
            m[(size_t)cy1 * J.cw + cx1] = 1;
        }
    }
    // block-aggregated append to the frame's guided work list: one atomic
    // per block (8 warps), warp offsets from a shared prefix
    __shared__ unsigned warpCount[8];
    __shared__ unsigned long long blockBase;
    const unsigned ballot = __ballot_sync(0xffffffffu, active);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    if (lane == 0)
        warpCount[warp] = __popc(ballot);
    __syncthreads();
    if (tid == 0) {
        unsigned total = 0;
        for (int w = 0; w < 8; ++w) {
            const unsigned c = warpCount[w];
            warpCount[w] = total;
            total += c;
        }
        blockBase = total ? atomicAdd(J.counters + kCntActiveOutput, (unsigned long long)total) : 0ull;
    }
    __syncthreads();
    if (active && J.listed) {
        const unsigned rank = warpCount[warp] + __popc(ballot & ((1u << lane) - 1u));
        J.actList[blockBase + rank] = ((uint32_t)oy << 16) | (uint32_t)ox;
    }
}

// Population count of a u8 plane region: counts chroma mask / trust mask.
__global__ void k_count(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart,
                        int njobs) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const size_t nc = (size_t)J.cw * J.ch;
    const size_t nm = (size_t)J.sw * J.sh;
    const size_t i = (size_t)tile * 1024 + threadIdx.x * 4;
    int c = 0, m = 0;
    for (int k = 0; k < 4; ++k) {
        if (i + k < nc) c += J.cmask[i + k] != 0;
        if (i + k < nm) m += J.mask[i + k] != 0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_down_sync(0xffffffffu, c, o);
        m += __shfl_down_sync(0xffffffffu, m, o);
    }
    __shared__ int sc[8], sm[8];
    if ((threadIdx.x & 31) == 0) {
        sc[threadIdx.x >> 5] = c;
        sm[threadIdx.x >> 5] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int tc = 0, tm = 0;
        for (int w = 0; w < 8; ++w) { tc += sc[w]; tm += sm[w]; }
        if (tc) atomicAdd(J.counters + kCntActiveChroma, (unsigned long long)tc);
        if (tm) atomicAdd(J.counters + kCntMaskPixels, (unsigned long long)tm);
    }
}

// ---------------------------------------------------------------------------
// Mutual-structure gate at chroma resolution. Gradients of lc, U, V are
// computed in shared memory for the tile plus a 4-pixel halo (the farthest
// any gate sample reaches), at clamped positions, exactly as the reference's
// dense Sobel rows; the sparse reference computes the same values wherever
// an active sample can read them.
// ---------------------------------------------------------------------------
constexpr int GT_X = 32, GT_Y = 8, GH = 4;

__global__ void __launch_bounds__(GT_X * GT_Y)
k_gate(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    __shared__ float src[3][GT_Y + 2 * GH + 2][GT_X + 2 * GH + 2];
    __shared__ float gx[3][GT_Y + 2 * GH][GT_X + 2 * GH];
    __shared__ float gy[3][GT_Y + 2 * GH][GT_X + 2 * GH];
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int w = J.cw, h = J.ch;
    const int tilesX = (w + GT_X - 1) / GT_X;
    const int x0 = (tile % tilesX) * GT_X, y0 = (tile / tilesX) * GT_Y;
    const int tid = threadIdx.y * GT_X + threadIdx.x;
    const int nthreads = GT_X * GT_Y;
    const float *planes[3] = { J.lc, J.U, J.V };
    constexpr int SW = GT_X + 2 * GH + 2, SH = GT_Y + 2 * GH + 2;
    for (int i = tid; i < 3 * SW * SH; i += nthreads) {
        const int p = i / (SW * SH), rem = i % (SW * SH);
        const int r = rem / SW, c = rem % SW;
        const int yy = iclamp(y0 - GH - 1 + r, 0, h - 1), xx = iclamp(x0 - GH - 1 + c, 0, w - 1);
        src[p][r][c] = ldf(planes[p] + (size_t)yy * w + xx);
    }
    __syncthreads();
    constexpr int GW = GT_X + 2 * GH, GHh = GT_Y + 2 * GH;
    for (int i = tid; i < 3 * GW * GHh; i += nthreads) {
        const int p = i / (GW * GHh), rem = i % (GW * GHh);
        const int r = rem / GW, c = rem % GW;
        const int yy = iclamp(y0 - GH + r, 0, h - 1), xx = iclamp(x0 - GH + c, 0, w - 1);
        const int sr = yy - y0 + GH + 1, sc = xx - x0 + GH + 1;
        const float tl = src[p][sr - 1][sc - 1], t = src[p][sr - 1][sc], tr = src[p][sr - 1][sc + 1];
        const float l = src[p][sr][sc - 1], rr = src[p][sr][sc + 1];
        const float bl = src[p][sr + 1][sc - 1], b = src[p][sr + 1][sc], br = src[p][sr + 1][sc + 1];
        gx[p][r][c] = (tr + 2.0f * rr + br - tl - 2.0f * l - bl) * 0.125f;
        gy[p][r][c] = (bl + 2.0f * b + br - tl - 2.0f * t - tr) * 0.125f;
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= w || y >= h)
        return;
    const size_t o = (size_t)y * w + x;
    const bool dense = !J.sparse ||
        (unsigned long long)J.counters[kCntActiveChroma] * 2ull >= (unsigned long long)w * h;
    if (!dense && J.cmask[o] == 0) {
        J.ms[o] = 0.0f;
        return;
    }
    // slot of a clamped coordinate
    auto sx = [&](int xx) { return iclamp(xx, 0, w - 1) - x0 + GH; };
    auto sy = [&](int yy) { return iclamp(yy, 0, h - 1) - y0 + GH; };
    float sxx = 0.0f, sxy = 0.0f, syy = 0.0f;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            const float a = gx[0][sy(y + dy)][sx(x + dx)];
            const float b = gy[0][sy(y + dy)][sx(x + dx)];
            sxx += a * a; sxy += a * b; syy += b * b;
        }
    const float jsum = sxx + syy;
    if (jsum < 1e-10f) {
        J.ms[o] = 0.0f;
        return;
    }
    const TensorDir dir = principalDirection(sxx, sxy, syy);
    const float nx = dir.nx, ny = dir.ny;
    float sumY = 0, sqY = 0, momY = 0, sumC = 0, sqC = 0, momC = 0;
    for (int k = -3; k <= 3; ++k) {
        const float px = (float)x + (float)k * nx;
        const float py = (float)y + (float)k * ny;
        const float fpx = floorf(px), fpy = floorf(py);
        const int rawX = (int)fpx, rawY = (int)fpy;
        const int bx0 = sx(rawX), bx1 = sx(rawX + 1);
        const int by0 = sy(rawY), by1 = sy(rawY + 1);
        const float fx = px - fpx, fy = py - fpy;
        float s[3];
        for (int p = 0; p < 3; ++p) {
            const float a = gx[p][by0][bx0] * nx + gy[p][by0][bx0] * ny;
            const float b = gx[p][by0][bx1] * nx + gy[p][by0][bx1] * ny;
            const float c = gx[p][by1][bx0] * nx + gy[p][by1][bx0] * ny;
            const float d = gx[p][by1][bx1] * nx + gy[p][by1][bx1] * ny;
            s[p] = a + (b - a) * fx + (c - a) * fy + (a - b - c + d) * fx * fy;
        }
        const float gY = fabsf(s[0]);
        const float gC = sqrtf(s[1] * s[1] + s[2] * s[2]);
        sumY += gY; sqY += gY * gY; momY += (float)k * gY;
        sumC += gC; sqC += gC * gC; momC += (float)k * gC;
    }
    if (sumY < 1e-9f || sumC < 1e-9f) {
        J.ms[o] = 0.0f;
        return;
    }
    const float partY = sumY * sumY / (sqY + 1e-12f);
    const float partC = sumC * sumC / (sqC + 1e-12f);
    const float ratio = partC / (partY + 1e-6f);
    const float dcent = fabsf(momY / sumY - momC / sumC);
    const float tw = sclamp((1.6f - ratio) / 0.4f, 0.0f, 1.0f);
    const float tp = sclamp((1.0f - dcent) / 0.5f, 0.0f, 1.0f);
    J.ms[o] = (tw * tw * (3.0f - 2.0f * tw)) * (tp * tp * (3.0f - 2.0f * tp));
}

} // namespace lgcr_b200
