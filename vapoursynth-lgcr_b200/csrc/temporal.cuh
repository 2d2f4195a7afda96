// TRecon temporal taps of the guided pass (reconstructChromaImpl,
// src/recon.cpp:642-745): each motion-compensated neighbour contributes its
// chroma sample nearest the mapped position, weighted by block confidence,
// a luma similarity (footprint level for static blocks, a box straddle test
// against the source luma for moving ones), the lanczos base kernel at the
// true offset and the phase-novelty factor of moving blocks.
#pragma once

#include "recon.cuh"

namespace lgcr_b200 {

// Accumulators and chroma hull carried through the temporal taps by value.
struct TemporalAcc {
    double u, v, wsum, sumAbs;
    float mnU, mxU, mnV, mxV;
};

// kernelEval(Lanczos) of src/lgcr.h:53-74 in double: sinc(x) sinc(x / taps)
// for |x| < taps, sinc(x) = sin(pi x) / (pi x) with sinc(0) = 1.
__device__ __forceinline__ double sincD(double x) {
    if (fabs(x) < 1e-8)
        return 1.0;
    x *= 3.14159265358979323846;
    return sin(x) / x;
}

__device__ __forceinline__ double lanczosD(double x, double taps) {
    x = fabs(x);
    return x < taps ? sincD(x) * sincD(x / taps) : 0.0;
}

// Kept out of line: Recon frames never take this path, and the guided
// kernel's register allocation stays that of the spatial taps.
static __device__ __noinline__ TemporalAcc temporalTaps(const FrameJob &J, int ox, int oy,
                                                        float L0, float scx, float scy,
                                                        float sigLoc, float guideFade,
                                                        float ssRamp, TemporalAcc t) {
    const int lx = iclamp((int)__ldg(J.ax.lpos + ox), 0, J.sw - 1);
    const int ly = iclamp((int)__ldg(J.ay.lpos + oy), 0, J.sh - 1);
    const float frw = J.rwF, frh = J.rhF;
    for (int k = 0; k < J.tnbCount; ++k) {
        const TemporalView &nb = J.tnb[k];
        const int bxx = min(nb.bw - 1, lx / 16);
        const int byy = min(nb.bh - 1, ly / 16);
        const size_t bi = (size_t)byy * nb.bw + bxx;
        const float tconf = ldf(nb.conf + bi);
        if (tconf < 0.05f)
            continue;
        const int imx = __ldg(nb.mvx + bi), imy = __ldg(nb.mvy + bi);
        const float mx = (float)imx, my = (float)imy;
        // nearest neighbour chroma sample to the mapped position
        const int tnx = iclamp((int)lroundf(scx + mx / frw), 0, J.cw - 1);
        const int tny = iclamp((int)lroundf(scy + my / frh), 0, J.ch - 1);
        const float ddx = ((float)tnx - scx) * frw - mx;
        const float ddy = ((float)tny - scy) * frh - my;
        const bool staticBlk = (fabsf(mx) + fabsf(my) <= 1.0f) && tconf > 0.5f;
        const size_t to = (size_t)tny * J.cw + tnx;
        float dL;
        if (staticBlk) {
            dL = ldf(nb.lc + to) - L0;
        } else {
            // footprint-straddle test against the source luma
            const double lxd = ((double)tnx + 0.5) * J.rw - 0.5 + J.shiftXd - (double)mx;
            const double lyd = ((double)tny + 0.5) * J.rh - 0.5 + J.shiftYd - (double)my;
            const int x0 = (int)ceil(lxd - 0.5 * J.rw), x1 = (int)ceil(lxd + 0.5 * J.rw);
            const int y0 = (int)ceil(lyd - 0.5 * J.rh), y1 = (int)ceil(lyd + 0.5 * J.rh);
            float md = 0.0f;
            for (int jj = y0; jj < y1; ++jj) {
                const float *row = J.Y + (size_t)iclamp(jj, 0, J.sh - 1) * J.sw;
                for (int ii = x0; ii < x1; ++ii)
                    md = smax(md, fabsf(ldf(row + iclamp(ii, 0, J.sw - 1)) - L0));
            }
            dL = md;
        }
        const float sigT = staticBlk ? sigLoc : 0.5f * sigLoc;
        const float simRaw = 1.0f / (1.0f + dL * dL / (sigT * sigT));
        const float sim = staticBlk ? 1.0f - guideFade * (1.0f - simRaw) : simRaw;
        const float kw = (float)(lanczosD((double)fabsf(ddx) / J.rw * (double)J.invWxC, J.support) *
                                 lanczosD((double)fabsf(ddy) / J.rh * (double)J.invWyC, J.support));
        float nw = 1.0f;
        if (!staticBlk) {
            nw = smax(ldf(J.tnwX + imx + 64), ldf(J.tnwY + imy + 64));
            nw *= 1.0f - ssRamp;
        }
        const float w = tconf * sim * kw * nw;
        const float u = ldf(nb.U + to), v = ldf(nb.V + to);
        const double wd = (double)w;
        t.u = fma(wd, (double)u, t.u);
        t.v = fma(wd, (double)v, t.v);
        t.wsum += wd;
        t.sumAbs += fabs(wd);
        t.mnU = runMin(t.mnU, u);
        t.mxU = runMax(t.mxU, u);
        t.mnV = runMin(t.mnV, v);
        t.mxV = runMax(t.mxV, v);
    }
    return t;
}

} // namespace lgcr_b200
