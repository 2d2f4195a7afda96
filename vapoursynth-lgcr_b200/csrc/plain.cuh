// Plain (unguided) reconstruction of one or two chroma-resolution planes at
// one output sample. Shared by the chroma base (two planes) and the algo 6
// detail map (degraded luma, one plane) so both use identical arithmetic:
//   separable   plainChromaSeparable (scalar)   src/recon.cpp:1151-1461
//   bilinear    plainChromaBilinear             src/recon.cpp:1031-1149
//   radial      plainChromaImpl<radial>         src/recon.cpp:828-1029
#pragma once

#include "recon.cuh"

namespace lgcr_b200 {

struct PlainCtx {
    const float *p0, *p1;        // p1 may be null (single plane)
    int w, h;                    // source plane size
    AxisView ax, ay;
    RadialView rad;
    int kernel, radial, clampHull;
    float margin, invWxC, invWyC, lutScale;
    int lutN;
    const float *lut;
    int noClampX, noClampY;      // every tap index of the axes is in range
    const double2 *uv;           // p0 / p1 as FP64 pairs (chroma), or null
};

__device__ __forceinline__ void plainSeparableAt(const PlainCtx &c, int ox, int oy, float &o0, float &o1) {
    const AxisView &ax = c.ax, &ay = c.ay;
    const int tx0 = __ldg(ax.start + ox), ty0 = __ldg(ay.start + oy);
    const float *wx = ax.w + (size_t)ox * ax.sup;
    const uint8_t *amx = ax.am + (size_t)ox * ax.sup;
    const float *wy = ay.w + (size_t)oy * ay.sup;
    const uint8_t *amy = ay.am + (size_t)oy * ay.sup;
    const bool dual = c.p1 != nullptr;
    double v0 = 0.0, v1 = 0.0;
    float mn0 = 1e30f, mx0 = -1e30f, mn1 = 1e30f, mx1 = -1e30f;
    for (int j = 0; j < ay.sup; ++j) {
        if (__ldg(amy + j) == 0)
            continue;
        const size_t rowOff = (size_t)iclamp(ty0 + j, 0, c.h - 1) * c.w;
        double h0 = 0.0, h1 = 0.0;
        float hmn0 = 1e30f, hmx0 = -1e30f, hmn1 = 1e30f, hmx1 = -1e30f;
        for (int i = 0; i < ax.sup; ++i) {
            if (__ldg(amx + i) == 0)
                continue;
            const size_t o = rowOff + iclamp(tx0 + i, 0, c.w - 1);
            const double wgt = (double)__ldg(wx + i);
            const float a = ldf(c.p0 + o);
            h0 = fma(wgt, (double)a, h0);
            hmn0 = smin(hmn0, a); hmx0 = smax(hmx0, a);
            if (dual) {
                const float b = ldf(c.p1 + o);
                h1 = fma(wgt, (double)b, h1);
                hmn1 = smin(hmn1, b); hmx1 = smax(hmx1, b);
            }
        }
        const double wgt = (double)__ldg(wy + j);
        v0 = fma(wgt, (double)(float)h0, v0);
        mn0 = smin(mn0, hmn0); mx0 = smax(mx0, hmx0);
        if (dual) {
            v1 = fma(wgt, (double)(float)h1, v1);
            mn1 = smin(mn1, hmn1); mx1 = smax(mx1, hmx1);
        }
    }
    const double ws = (double)__ldg(ax.wsum + ox) * (double)__ldg(ay.wsum + oy);
    const double wa = (double)__ldg(ax.wabs + ox) * (double)__ldg(ay.wabs + oy);
    if (ws > 1e-6 && ws >= 0.05 * wa) {
        v0 /= ws;
        v1 /= ws;
    } else {
        const float px = __ldg(ax.pos + ox), py = __ldg(ay.pos + oy);
        v0 = bilinearAt(c.p0, c.w, c.h, px, py);
        if (dual)
            v1 = bilinearAt(c.p1, c.w, c.h, px, py);
    }
    if (c.clampHull) {
        v0 = sclamp(v0, (double)(mn0 - c.margin), (double)(mx0 + c.margin));
        if (dual)
            v1 = sclamp(v1, (double)(mn1 - c.margin), (double)(mx1 + c.margin));
    }
    o0 = (float)v0;
    o1 = (float)v1;
}

__device__ __forceinline__ const float *radialWeightsAt(const RadialView &r, int ox, int oy) {
    if (!r.valid)
        return nullptr;
    const size_t phase = (size_t)__ldg(r.yPhase + oy) * r.phasesX + __ldg(r.xPhase + ox);
    return r.weights + phase * (size_t)r.supX * r.supY;
}

// Radial plain base with the phase table, taps in range and an even support
// SUP: the loop of plainRadialAt fully unrolled, tap activity from bit
// masks, weight pairs as 8-byte loads; the same sums in the same order.
template <int SUP>
__device__ __forceinline__ void plainRadialTable(const PlainCtx &c, int ox, int oy, const float *base,
                                                 float &o0, float &o1) {
    const AxisView &ax = c.ax, &ay = c.ay;
    const int tx0 = __ldg(ax.start + ox), ty0 = __ldg(ay.start + oy);
    uint32_t mx = 0, my = 0;
#pragma unroll
    for (int i = 0; i < SUP; ++i) {
        mx |= (__ldg(ax.am + (size_t)ox * SUP + i) != 0 ? 1u : 0u) << i;
        my |= (__ldg(ay.am + (size_t)oy * SUP + i) != 0 ? 1u : 0u) << i;
    }
    const float scx = __ldg(ax.pos + ox), scy = __ldg(ay.pos + oy);
    const bool dual = c.p1 != nullptr;
    double acc0 = 0.0, acc1 = 0.0, wsum = 0.0, sumAbs = 0.0;
    float mn0 = 1e30f, mx0 = -1e30f, mn1 = 1e30f, mx1 = -1e30f;
    if (dual && c.uv) {
        // both planes from the FP64 pairs: one conversion per tap (the
        // weight); the hull compares the exact double copies of the samples
        double n0 = (double)mn0, x0d = (double)mx0, n1 = (double)mn1, x1d = (double)mx1;
#pragma unroll
        for (int j = 0; j < SUP; ++j) {
            if (!((my >> j) & 1u))
                continue;
            const double2 *r = c.uv + (size_t)(ty0 + j) * c.w + tx0;
            const float2 *wrow = reinterpret_cast<const float2 *>(base + j * SUP);
#pragma unroll
            for (int q = 0; q < SUP / 2; ++q) {
                const float2 w2 = __ldg(wrow + q);
                const float wk[2] = { w2.x, w2.y };
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int i = 2 * q + h;
                    if (!((mx >> i) & 1u))
                        continue;
                    const double wd = (double)wk[h];
                    const double2 p = __ldg(r + i);
                    acc0 = fma(wd, p.x, acc0);
                    wsum += wd;
                    sumAbs += fabs(wd);
                    n0 = smin(n0, p.x); x0d = smax(x0d, p.x);
                    acc1 = fma(wd, p.y, acc1);
                    n1 = smin(n1, p.y); x1d = smax(x1d, p.y);
                }
            }
        }
        mn0 = (float)n0; mx0 = (float)x0d; mn1 = (float)n1; mx1 = (float)x1d;
    } else {
#pragma unroll
    for (int j = 0; j < SUP; ++j) {
        if (!((my >> j) & 1u))
            continue;
        const float *r0 = c.p0 + (size_t)(ty0 + j) * c.w + tx0;
        const float *r1 = dual ? c.p1 + (size_t)(ty0 + j) * c.w + tx0 : nullptr;
        const float2 *wrow = reinterpret_cast<const float2 *>(base + j * SUP);
#pragma unroll
        for (int q = 0; q < SUP / 2; ++q) {
            const float2 w2 = __ldg(wrow + q);
            const float wk[2] = { w2.x, w2.y };
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = 2 * q + h;
                if (!((mx >> i) & 1u))
                    continue;
                const float weight = wk[h];
                const float a = ldf(r0 + i);
                acc0 = fma((double)weight, (double)a, acc0);
                wsum += (double)weight;
                sumAbs += (double)fabsf(weight);
                mn0 = smin(mn0, a); mx0 = smax(mx0, a);
                if (dual) {
                    const float b = ldf(r1 + i);
                    acc1 = fma((double)weight, (double)b, acc1);
                    mn1 = smin(mn1, b); mx1 = smax(mx1, b);
                }
            }
        }
    }
    }
    double v0, v1 = 0.0;
    if (wsum > 1e-6 && wsum >= 0.05 * sumAbs) {
        v0 = acc0 / wsum;
        if (dual) v1 = acc1 / wsum;
    } else {
        v0 = bilinearAt(c.p0, c.w, c.h, scx, scy);
        if (dual) v1 = bilinearAt(c.p1, c.w, c.h, scx, scy);
    }
    if (c.clampHull) {
        v0 = sclamp(v0, (double)(mn0 - c.margin), (double)(mx0 + c.margin));
        if (dual) v1 = sclamp(v1, (double)(mn1 - c.margin), (double)(mx1 + c.margin));
    }
    o0 = (float)v0;
    o1 = (float)v1;
}

__device__ __forceinline__ void plainRadialAt(const PlainCtx &c, int ox, int oy, float &o0, float &o1) {
    const AxisView &ax = c.ax, &ay = c.ay;
    const int tx0 = __ldg(ax.start + ox), ty0 = __ldg(ay.start + oy);
    const uint8_t *amx = ax.am + (size_t)ox * ax.sup;
    const uint8_t *amy = ay.am + (size_t)oy * ay.sup;
    const float scx = __ldg(ax.pos + ox), scy = __ldg(ay.pos + oy);
    const float *base = radialWeightsAt(c.rad, ox, oy);
    if (base && c.noClampX && c.noClampY && ax.sup == ay.sup && c.rad.supX == ax.sup &&
        c.rad.supY == ay.sup) {
        switch (ax.sup) {
        case 4: plainRadialTable<4>(c, ox, oy, base, o0, o1); return;
        case 6: plainRadialTable<6>(c, ox, oy, base, o0, o1); return;
        case 8: plainRadialTable<8>(c, ox, oy, base, o0, o1); return;
        default: break;
        }
    }
    const bool dual = c.p1 != nullptr;
    double acc0 = 0.0, acc1 = 0.0, wsum = 0.0, sumAbs = 0.0;
    float mn0 = 1e30f, mx0 = -1e30f, mn1 = 1e30f, mx1 = -1e30f;
    for (int j = 0; j < ay.sup; ++j) {
        if (__ldg(amy + j) == 0)
            continue;
        const size_t rowOff = (size_t)iclamp(ty0 + j, 0, c.h - 1) * c.w;
        const float dy = ((float)(ty0 + j) - scy) * c.invWyC;
        for (int i = 0; i < ax.sup; ++i) {
            if (__ldg(amx + i) == 0)
                continue;
            const size_t o = rowOff + iclamp(tx0 + i, 0, c.w - 1);
            float weight;
            if (base) {
                weight = ldf(base + (size_t)j * ax.sup + i);
            } else {
                const float dx = ((float)(tx0 + i) - scx) * c.invWxC;
                weight = lutLookupDev(c.lut, c.lutN, sqrtf(dx * dx + dy * dy) * c.lutScale);
            }
            const float a = ldf(c.p0 + o);
            acc0 = fma((double)weight, (double)a, acc0);
            wsum += (double)weight;
            sumAbs += (double)fabsf(weight);
            mn0 = smin(mn0, a); mx0 = smax(mx0, a);
            if (dual) {
                const float b = ldf(c.p1 + o);
                acc1 = fma((double)weight, (double)b, acc1);
                mn1 = smin(mn1, b); mx1 = smax(mx1, b);
            }
        }
    }
    double v0, v1 = 0.0;
    if (wsum > 1e-6 && wsum >= 0.05 * sumAbs) {
        v0 = acc0 / wsum;
        if (dual) v1 = acc1 / wsum;
    } else {
        v0 = bilinearAt(c.p0, c.w, c.h, scx, scy);
        if (dual) v1 = bilinearAt(c.p1, c.w, c.h, scx, scy);
    }
    if (c.clampHull) {
        v0 = sclamp(v0, (double)(mn0 - c.margin), (double)(mx0 + c.margin));
        if (dual) v1 = sclamp(v1, (double)(mn1 - c.margin), (double)(mx1 + c.margin));
    }
    o0 = (float)v0;
    o1 = (float)v1;
}

__device__ __forceinline__ void plainAt(const PlainCtx &c, int ox, int oy, float &o0, float &o1) {
    if (c.radial) {
        plainRadialAt(c, ox, oy, o0, o1);
    } else if (c.kernel == 0) {
        const int x0 = __ldg(c.ax.cbI0 + ox), y0 = __ldg(c.ay.cbI0 + oy);
        const float fx = __ldg(c.ax.cbF + ox), fy = __ldg(c.ay.cbF + oy);
        o0 = bilinearFast(c.p0, c.w, c.h, x0, fx, y0, fy);
        o1 = c.p1 ? bilinearFast(c.p1, c.w, c.h, x0, fx, y0, fy) : 0.0f;
    } else {
        plainSeparableAt(c, ox, oy, o0, o1);
    }
}

// Context for the two-plane chroma base of a frame.
__device__ __forceinline__ PlainCtx chromaPlainCtx(const FrameJob &J) {
    PlainCtx c;
    c.p0 = J.U; c.p1 = J.V; c.w = J.cw; c.h = J.ch;
    c.ax = J.ax; c.ay = J.ay; c.rad = J.rad;
    c.kernel = J.kernel; c.radial = J.radial; c.clampHull = J.clampHull;
    c.margin = J.margin; c.invWxC = J.invWxC; c.invWyC = J.invWyC;
    c.lutScale = J.lutScale; c.lutN = J.lutN; c.lut = J.lut;
    c.noClampX = J.noClampX; c.noClampY = J.noClampY;
    c.uv = reinterpret_cast<const double2 *>(J.uvd);
    return c;
}

} // namespace lgcr_b200
