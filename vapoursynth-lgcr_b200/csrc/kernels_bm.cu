// Collaborative block refinement and 4:2:0 back-projection.
//   k_bm_group      per 8-px anchor: 25-candidate search on a (luma, chroma)
//                   cost, best 4 under the match limit, 2D Haar per patch,
//                   1D Haar across the group, hard threshold (DC kept),
//                   inverse, hull clamp         collaborativeChromaFilter
//                                               src/bm.cpp:250-418 (helpers 13-246)
//   k_bm_aggregate  per output pixel: windowed weighted sum of every group
//                   patch covering it, added in anchor order (the reference's
//                   sequential += order), then src + 0.65 (filtered - src)
//                                               src/bm.cpp:393-437
//   k_backproject   per chroma sample: r = src - mean(2x2 out); out += bp r,
//                   stored to the typed output (the last stage)
//                                               src/algos.cpp:663-677
#include "kernels.cuh"

namespace lgcr_b200 {

constexpr int kPatch = 8, kGroup = 4;
constexpr float kInvSqrt2 = 0.7071067811865475f;
constexpr int kAnchorFloats = 2 * kGroup * 64 + 8;   // filtered U/V + group weight
constexpr int kAnchorInts = 1 + 2 * kGroup;          // group size + match coords

__device__ __constant__ float kWindow[8] = {0.25f, 0.50f, 0.75f, 1.0f, 1.0f, 0.75f, 0.50f, 0.25f};

// guide sample at output coordinates: source luma, bilinearly resized with
// double positions when the output size differs (bm.cpp:255-268)
__device__ __forceinline__ float bmGuide(const FrameJob &J, int x, int y) {
    if (J.sameSize)
        return ldf(J.Y + (size_t)y * J.sw + x);
    const double sx = (double)J.sw / J.W, sy = (double)J.sh / J.H;
    const double gx = (x + 0.5) * sx - 0.5, gy = (y + 0.5) * sy - 0.5;
    const double fx0 = floor(gx), fy0 = floor(gy);
    const int x0 = (int)fx0, y0 = (int)fy0;
    const float fx = (float)(gx - x0), fy = (float)(gy - y0);
    const int xa = iclamp(x0, 0, J.sw - 1), xb = iclamp(x0 + 1, 0, J.sw - 1);
    const int ya = iclamp(y0, 0, J.sh - 1), yb = iclamp(y0 + 1, 0, J.sh - 1);
    const float a = ldf(J.Y + (size_t)ya * J.sw + xa), b = ldf(J.Y + (size_t)ya * J.sw + xb);
    const float c = ldf(J.Y + (size_t)yb * J.sw + xa), d = ldf(J.Y + (size_t)yb * J.sw + xb);
    return a + (b - a) * fx + (c - a) * fy + (a - b - c + d) * fx * fy;
}

__device__ __forceinline__ void haarFwd(float *v, int count) {
    float t[8];
    for (int length = count; length > 1; length /= 2) {
        const int half = length / 2;
        for (int i = 0; i < half; ++i) {
            const float a = v[2 * i], b = v[2 * i + 1];
            t[i] = (a + b) * kInvSqrt2;
            t[half + i] = (a - b) * kInvSqrt2;
        }
        for (int i = 0; i < length; ++i) v[i] = t[i];
    }
}

__device__ __forceinline__ void haarInv(float *v, int count) {
    float t[8];
    for (int length = 2; length <= count; length *= 2) {
        const int half = length / 2;
        for (int i = 0; i < half; ++i) {
            const float a = v[i], b = v[half + i];
            t[2 * i] = (a + b) * kInvSqrt2;
            t[2 * i + 1] = (a - b) * kInvSqrt2;
        }
        for (int i = 0; i < length; ++i) v[i] = t[i];
    }
}

__device__ __forceinline__ int anchorCount(const FrameJob &J) { return J.bmAnchorsX * J.bmAnchorsY; }

// One warp per anchor, 8 anchors per block.
__global__ void __launch_bounds__(256)
k_bm_group(LGCR_STAGE_ARGS) {
    __shared__ float grp[8][2][64 * kGroup];        // [plane][offset*4 + k]
    __shared__ float costs[8][32];
    __shared__ int cbx[8][32], cby[8][32];
    __shared__ int meta[8][kAnchorInts];
    __shared__ float bestC[8][kGroup];
    __shared__ int bestX[8][kGroup], bestY[8][kGroup];
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int anchor = (blockIdx.x - tileStart[f]) * 8 + warp;
    if (anchor >= anchorCount(J))
        return;                                      // whole warp leaves together
    const int W = J.W, H = J.H;
    const int ay = __ldg(J.bmStartsY + anchor / J.bmAnchorsX);
    const int ax = __ldg(J.bmStartsX + anchor % J.bmAnchorsX);
    const float *U = J.oU, *V = J.oV;
    // candidate grid: dy outer, dx inner, steps of 4 over [-8, 8]
    if (lane < 25) {
        const int dy = -8 + 4 * (lane / 5), dx = -8 + 4 * (lane % 5);
        const int bx = iclamp(ax + dx, 0, W - kPatch), by = iclamp(ay + dy, 0, H - kPatch);
        cbx[warp][lane] = bx;
        cby[warp][lane] = by;
        float cost = 0.0f;
        if (!(bx == ax && by == ay)) {
            int samples = 0;
            for (int py = 0; py < kPatch; py += 2)
                for (int px = 0; px < kPatch; px += 2) {
                    const float dg = bmGuide(J, ax + px, ay + py) - bmGuide(J, bx + px, by + py);
                    const size_t oa = (size_t)(ay + py) * W + ax + px;
                    const size_t ob = (size_t)(by + py) * W + bx + px;
                    const float du = U[oa] - U[ob];
                    const float dv = V[oa] - V[ob];
                    cost += dg * dg + 0.25f * (du * du + dv * dv);
                    ++samples;
                }
            cost = cost / (float)samples;
        }
        costs[warp][lane] = cost;
    }
    __syncwarp();
    // The reference walks the candidates in enumeration order, skips a
    // position seen before and inserts the rest into a best-4 list that keeps
    // an earlier candidate ahead of a later one of equal cost: the list holds
    // the 4 smallest kept candidates by (cost, enumeration index). Each lane
    // finds whether its candidate is kept and its rank among the kept ones.
    bool keep = false;
    float myCost = 0.0f;
    int myBx = 0, myBy = 0;
    if (lane < 25) {
        myBx = cbx[warp][lane];
        myBy = cby[warp][lane];
        myCost = costs[warp][lane];
        keep = true;
        for (int i = 0; i < lane; ++i)
            if (cbx[warp][i] == myBx && cby[warp][i] == myBy) {
                keep = false;
                break;
            }
    }
    const unsigned kept = __ballot_sync(0xffffffffu, keep);
    if (keep) {
        int rank = 0;
        for (int d = 0; d < 25; ++d) {
            if (d == lane || !((kept >> d) & 1u))
                continue;
            const float cd = costs[warp][d];
            if (cd < myCost || (cd == myCost && d < lane))
                ++rank;
        }
        if (rank < kGroup) {
            bestC[warp][rank] = myCost;
            bestX[warp][rank] = myBx;
            bestY[warp][rank] = myBy;
        }
    }
    __syncwarp();
    if (lane == 0) {
        const int count = min(__popc(kept), kGroup);
        const float gs = J.bmSigma;
        const float matchLimit = smax(4e-5f, 4.0f * gs * gs);
        int eligible = 0;
        while (eligible < count && bestC[warp][eligible] <= matchLimit)
            ++eligible;
        const int groupCount = eligible >= 4 ? 4 : (eligible >= 2 ? 2 : 1);
        meta[warp][0] = groupCount < 2 ? 0 : groupCount;
        for (int k = 0; k < kGroup; ++k) {
            meta[warp][1 + 2 * k] = k < count ? bestX[warp][k] : 0;
            meta[warp][2 + 2 * k] = k < count ? bestY[warp][k] : 0;
        }
    }
    __syncwarp();
    int *gout = J.bmGroups + (size_t)anchor * kAnchorInts;
    const int groupCount = meta[warp][0];
    if (lane < kAnchorInts)
        gout[lane] = meta[warp][lane];
    if (groupCount == 0)
        return;
    // load group patches
    for (int i = lane; i < groupCount * 64; i += 32) {
        const int k = i / 64, off = i % 64;
        const int bx = meta[warp][1 + 2 * k], by = meta[warp][2 + 2 * k];
        const size_t o = (size_t)(by + off / 8) * W + bx + off % 8;
        grp[warp][0][off * kGroup + k] = U[o];
        grp[warp][1][off * kGroup + k] = V[o];
    }
    __syncwarp();
    // per-offset hull of the group
    float hull[2][2][2];   // [plane][min/max][2 offsets per lane]
    for (int j = 0; j < 2; ++j) {
        const int off = lane + 32 * j;
        for (int p = 0; p < 2; ++p) {
            float mn = INFINITY, mx = -INFINITY;
            for (int k = 0; k < groupCount; ++k) {
                const float v = grp[warp][p][off * kGroup + k];
                mn = smin(mn, v); mx = smax(mx, v);
            }
            hull[p][0][j] = mn; hull[p][1][j] = mx;
        }
    }
    // forward 2D Haar per patch: rows, then columns
    const int tasks = 2 * groupCount * 8;
    for (int t = lane; t < tasks; t += 32) {
        const int p = t / (groupCount * 8), rem = t % (groupCount * 8), k = rem / 8, r = rem % 8;
        float v[8];
        for (int i = 0; i < 8; ++i) v[i] = grp[warp][p][(r * 8 + i) * kGroup + k];
        haarFwd(v, 8);
        for (int i = 0; i < 8; ++i) grp[warp][p][(r * 8 + i) * kGroup + k] = v[i];
    }
    __syncwarp();
    for (int t = lane; t < tasks; t += 32) {
        const int p = t / (groupCount * 8), rem = t % (groupCount * 8), k = rem / 8, c = rem % 8;
        float v[8];
        for (int i = 0; i < 8; ++i) v[i] = grp[warp][p][(i * 8 + c) * kGroup + k];
        haarFwd(v, 8);
        for (int i = 0; i < 8; ++i) grp[warp][p][(i * 8 + c) * kGroup + k] = v[i];
    }
    __syncwarp();
    // across the group: forward, hard threshold (DC of the first kept), inverse
    const float sigma = sclamp(0.6f * J.bmSigma, 0.002f, 0.012f);
    const float threshold = 2.7f * sigma;
    int retained = 0;
    for (int t = lane; t < 64; t += 32) {
        for (int p = 0; p < 2; ++p) {
            float v[4];
            for (int k = 0; k < kGroup; ++k) v[k] = grp[warp][p][t * kGroup + k];
            haarFwd(v, groupCount);
            for (int k = 0; k < groupCount; ++k) {
                const bool keepDC = t == 0 && k == 0;
                if (!keepDC && fabsf(v[k]) < threshold) v[k] = 0.0f;
                else ++retained;
            }
            haarInv(v, groupCount);
            for (int k = 0; k < groupCount; ++k) grp[warp][p][t * kGroup + k] = v[k];
        }
    }
    for (int o = 16; o > 0; o >>= 1)
        retained += __shfl_down_sync(0xffffffffu, retained, o);
    __syncwarp();
    // inverse 2D Haar: columns, then rows
    for (int t = lane; t < tasks; t += 32) {
        const int p = t / (groupCount * 8), rem = t % (groupCount * 8), k = rem / 8, c = rem % 8;
        float v[8];
        for (int i = 0; i < 8; ++i) v[i] = grp[warp][p][(i * 8 + c) * kGroup + k];
        haarInv(v, 8);
        for (int i = 0; i < 8; ++i) grp[warp][p][(i * 8 + c) * kGroup + k] = v[i];
    }
    __syncwarp();
    for (int t = lane; t < tasks; t += 32) {
        const int p = t / (groupCount * 8), rem = t % (groupCount * 8), k = rem / 8, r = rem % 8;
        float v[8];
        for (int i = 0; i < 8; ++i) v[i] = grp[warp][p][(r * 8 + i) * kGroup + k];
        haarInv(v, 8);
        for (int i = 0; i < 8; ++i) grp[warp][p][(r * 8 + i) * kGroup + k] = v[i];
    }
    __syncwarp();
    float *pout = J.bmPatch + (size_t)anchor * kAnchorFloats;
    for (int j = 0; j < 2; ++j) {
        const int off = lane + 32 * j;
        for (int p = 0; p < 2; ++p)
            for (int k = 0; k < groupCount; ++k)
                pout[(p * kGroup + k) * 64 + off] =
                    sclamp(grp[warp][p][off * kGroup + k], hull[p][0][j], hull[p][1][j]);
    }
    if (lane == 0)
        pout[2 * kGroup * 64] = 1.0f / (1.0f + (float)retained);
}

// first index in a sorted start list with value >= v
__device__ __forceinline__ int lowerBound(const int *a, int n, int v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__global__ void k_bm_aggregate(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int x, y;
    tile32x8(blockIdx.x - tileStart[f], J.W, x, y);
    if (x >= J.W || y >= J.H)
        return;
    // anchors whose matches can cover (x, y): match within +-8 of the anchor
    const int iy0 = lowerBound(J.bmStartsY, J.bmAnchorsY, y - 15);
    const int iy1 = lowerBound(J.bmStartsY, J.bmAnchorsY, y + 9);
    const int ix0 = lowerBound(J.bmStartsX, J.bmAnchorsX, x - 15);
    const int ix1 = lowerBound(J.bmStartsX, J.bmAnchorsX, x + 9);
    float su = 0.0f, sv = 0.0f, sw = 0.0f;
    for (int iy = iy0; iy < iy1; ++iy)
        for (int ix = ix0; ix < ix1; ++ix) {
            const int anchor = iy * J.bmAnchorsX + ix;
            const int *g = J.bmGroups + (size_t)anchor * kAnchorInts;
            const int groupCount = g[0];
            if (groupCount == 0)
                continue;
            const float *pv = J.bmPatch + (size_t)anchor * kAnchorFloats;
            const float gw = pv[2 * kGroup * 64];
            for (int k = 0; k < groupCount; ++k) {
                const int px = x - g[1 + 2 * k], py = y - g[2 + 2 * k];
                if (px < 0 || px >= kPatch || py < 0 || py >= kPatch)
                    continue;
                const float weight = gw * kWindow[px] * kWindow[py];
                const int off = py * kPatch + px;
                su += weight * pv[(0 * kGroup + k) * 64 + off];
                sv += weight * pv[(1 * kGroup + k) * 64 + off];
                sw += weight;
            }
        }
    const size_t o = (size_t)y * J.W + x;
    const float srcU = J.oU[o], srcV = J.oV[o];
    if (sw > 0.0f) {
        const float fu = su / sw, fv = sv / sw;
        J.oU[o] = srcU + 0.65f * (fu - srcU);
        J.oV[o] = srcV + 0.65f * (fv - srcV);
    }
}

__global__ void k_backproject(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int cx, cy;
    tile32x8(blockIdx.x - tileStart[f], J.cw, cx, cy);
    if (cx >= J.cw || cy >= J.ch)
        return;
    const int x0 = 2 * cx, y0 = 2 * cy, W = J.W;
    const float bp = J.bpGain;
    float *planes[2] = { J.oU, J.oV };
    const float *srcs[2] = { J.U, J.V };
    for (int p = 0; p < 2; ++p) {
        float *o = planes[p];
        const float p00 = o[(size_t)y0 * W + x0], p10 = o[(size_t)y0 * W + x0 + 1];
        const float p01 = o[(size_t)(y0 + 1) * W + x0], p11 = o[(size_t)(y0 + 1) * W + x0 + 1];
        const float r = ldf(srcs[p] + (size_t)cy * J.cw + cx) - 0.25f * (p00 + p10 + p01 + p11);
        const float d = bp * r;
        if (J.bpStores) {
            // the last stage: the final samples go to the typed output
            storeChroma(J, 1 + p, x0, y0, p00 + d);
            storeChroma(J, 1 + p, x0 + 1, y0, p10 + d);
            storeChroma(J, 1 + p, x0, y0 + 1, p01 + d);
            storeChroma(J, 1 + p, x0 + 1, y0 + 1, p11 + d);
            continue;
        }
        o[(size_t)y0 * W + x0] = p00 + d;
        o[(size_t)y0 * W + x0 + 1] = p10 + d;
        o[(size_t)(y0 + 1) * W + x0] = p01 + d;
        o[(size_t)(y0 + 1) * W + x0 + 1] = p11 + d;
    }
}

} // namespace lgcr_b200
