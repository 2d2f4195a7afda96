// Chroma reconstruction stage: one thread per output pixel.
//   plain separable   plainChromaSeparable (scalar)   src/recon.cpp:1151-1461
//   plain bilinear    plainChromaBilinear             src/recon.cpp:1031-1149
//   plain radial      plainChromaImpl<radial>         src/recon.cpp:828-1029
//   guided            reconstructChromaImpl (scalar)  src/recon.cpp:14-819
//   luma resize       resampleH/V, resampleRadial     src/kernels.cpp:171-334
//   output store      floatToPlane                    src/lgcr.h:997-1013
// FP64 accumulators stay FP64 (B200 issues FP64 at half the FP32 rate); a
// product of two floats is exact in double, so fma(w, u, acc) rounds exactly
// like the reference's acc += double(w) * u.
#include "kernels.cuh"
#include "plain.cuh"

namespace lgcr_b200 {

__device__ __forceinline__ void plainPixel(const FrameJob &J, int ox, int oy, float &u, float &v) {
    plainAt(chromaPlainCtx(J), ox, oy, u, v);
}

// ---------------------------------------------------------------------------
// guided reconstruction (algo 2; the algo 4 selector variants reuse it)
// ---------------------------------------------------------------------------
struct Guided {
    double u, v;
    float L0, ssRamp, guideFade, nx, ny;
    bool hasDir;
};

__device__ __forceinline__ Guided guidedPixel(const FrameJob &J, int ox, int oy) {
    const AxisView &ax = J.ax, &ay = J.ay;
    const int sw = J.sw, sh = J.sh, cw = J.cw, ch = J.ch;
    Guided g;
    // guide metadata (prepareGuideRow, recon.cpp:155-220)
    const int bxi = __ldg(ax.lbI0 + ox), byi = __ldg(ay.lbI0 + oy);
    const float bxf = __ldg(ax.lbF + ox), byf = __ldg(ay.lbF + oy);
    const float L0 = bilinearFast(J.Y, sw, sh, bxi, bxf, byi, byf);
    const float jxx = bilinearFast(J.jxx, sw, sh, bxi, bxf, byi, byf);
    const float jxy = bilinearFast(J.jxy, sw, sh, bxi, bxf, byi, byf);
    const float jyy = bilinearFast(J.jyy, sw, sh, bxi, bxf, byi, byf);
    const float jsum = jxx + jyy;
    const TensorDir dir = principalDirection(jxx, jxy, jyy);
    const bool hasDir = jsum > 1e-6f;
    const float lx = __ldg(ax.lpos + ox), ly = __ldg(ay.lpos + oy);
    const float nx = dir.nx, ny = dir.ny;
    float minDiffN = 0.0f, ridgeRev = 0.0f;
    if (hasDir) {
        const float yA = bilinearAt(J.Y, sw, sh, lx - J.spOut * nx, ly - J.spOut * ny);
        const float yB = bilinearAt(J.Y, sw, sh, lx + J.spOut * nx, ly + J.spOut * ny);
        minDiffN = smin(fabsf(yA - L0), fabsf(yB - L0));
        if (J.ridge) {
            const float dl = 1.5f * J.spOut;
            const float ym2 = bilinearAt(J.Y, sw, sh, lx - 2.0f * dl * nx, ly - 2.0f * dl * ny);
            const float ym1 = bilinearAt(J.Y, sw, sh, lx - dl * nx, ly - dl * ny);
            const float yp1 = bilinearAt(J.Y, sw, sh, lx + dl * nx, ly + dl * ny);
            const float yp2 = bilinearAt(J.Y, sw, sh, lx + 2.0f * dl * nx, ly + 2.0f * dl * ny);
            const float diff[4] = { ym1 - ym2, L0 - ym1, yp1 - L0, yp2 - yp1 };
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const float a = diff[q], b = diff[q + 1];
                if (a > 0.0f && b < 0.0f)
                    ridgeRev = smax(ridgeRev, smin(a, -b));
                if (a < 0.0f && b > 0.0f)
                    ridgeRev = smax(ridgeRev, smin(-a, b));
            }
        }
    }
    const float scx = __ldg(ax.pos + ox), scy = __ldg(ay.pos + oy);
    const float fxp = scx - floorf(scx);
    const float fyp = scy - floorf(scy);
    const float phx = smin(fxp, 1.0f - fxp);
    const float phy = smin(fyp, 1.0f - fyp);
    const float phaseGate = (1.0f - 2.0f * phx) * (1.0f - 2.0f * phy);
    float mutualFade = 1.0f;
    if (J.useMs) {
        const float gate = bilinearFast(J.ms, cw, ch, __ldg(ax.cbI0 + ox), __ldg(ax.cbF + ox),
                                        __ldg(ay.cbI0 + oy), __ldg(ay.cbF + oy));
        mutualFade = 1.0f - J.msStrength * (1.0f - gate);
    }

    // pass 1: window luma range and chroma hull over active taps
    const int tx0 = __ldg(ax.start + ox), ty0 = __ldg(ay.start + oy);
    const float *wxp = ax.w + (size_t)ox * ax.sup;
    const uint8_t *amx = ax.am + (size_t)ox * ax.sup;
    const float *wyp = ay.w + (size_t)oy * ay.sup;
    const uint8_t *amy = ay.am + (size_t)oy * ay.sup;
    float maxAbsDL = 0.0f;
    float hMinU = 1e30f, hMaxU = -1e30f, hMinV = 1e30f, hMaxV = -1e30f;
    for (int j = 0; j < ay.sup; ++j) {
        if (__ldg(amy + j) == 0)
            continue;
        const size_t rowOff = (size_t)iclamp(ty0 + j, 0, ch - 1) * cw;
        for (int i = 0; i < ax.sup; ++i) {
            if (__ldg(amx + i) == 0)
                continue;
            const size_t o = rowOff + iclamp(tx0 + i, 0, cw - 1);
            const float l = ldf(J.lc + o), u = ldf(J.U + o), v = ldf(J.V + o);
            maxAbsDL = smax(maxAbsDL, fabsf(l - L0));
            hMinU = smin(hMinU, u); hMaxU = smax(hMaxU, u);
            hMinV = smin(hMinV, v); hMaxV = smax(hMaxV, v);
        }
    }

    const float t2 = sclamp(minDiffN / (0.1f * maxAbsDL + 1e-6f), 0.0f, 1.0f);
    const float ssRamp = t2 * t2 * (3.0f - 2.0f * t2);
    const float sigMult = J.sratio + (J.sdb - J.sratio) * ssRamp;
    const float sigLoc = smax(J.sigma, sigMult * maxAbsDL);
    const float invSigma2 = 1.0f / (sigLoc * sigLoc);
    const float ridgeFade = 1.0f - sclamp(2.0f * ridgeRev / (maxAbsDL + 1e-6f), 0.0f, 1.0f);
    float cedgeFade = 1.0f;
    if (J.cedge && hasDir) {
        // chroma-edge presence fade (recon.cpp:385-407)
        const float rcMax = smax(hMaxU - hMinU, hMaxV - hMinV);
        if (rcMax > 1e-6f) {
            float gmax = 0.0f;
            const float anx = fabsf(nx), any = fabsf(ny);
            for (int j = 0; j < ay.sup; ++j) {
                const int ty = iclamp(ty0 + j, 0, ch - 1);
                const int ty1 = min(ty + 1, ch - 1);
                for (int i = 0; i < ax.sup; ++i) {
                    const int tx = iclamp(tx0 + i, 0, cw - 1);
                    const int tx1 = min(tx + 1, cw - 1);
                    const float u00 = ldf(J.U + (size_t)ty * cw + tx);
                    const float v00 = ldf(J.V + (size_t)ty * cw + tx);
                    const float gu = smax(fabsf(ldf(J.U + (size_t)ty * cw + tx1) - u00) * anx,
                                          fabsf(ldf(J.U + (size_t)ty1 * cw + tx) - u00) * any);
                    const float gv = smax(fabsf(ldf(J.V + (size_t)ty * cw + tx1) - v00) * anx,
                                          fabsf(ldf(J.V + (size_t)ty1 * cw + tx) - v00) * any);
                    gmax = smax(gmax, smax(gu, gv));
                }
            }
            const float wc = rcMax / (gmax + 1e-6f);
            cedgeFade = sclamp((2.2f - wc) / 0.7f, 0.0f, 1.0f);
        }
    }
    const float guideFade = ridgeFade * cedgeFade * mutualFade * J.strength;

    // phase-0 rescue with kappa^2 (recon.cpp:425-475)
    float rescue = 0.0f;
    {
        const int ncx = iclamp((int)lroundf(scx), 0, cw - 1);
        const int ncy = iclamp((int)lroundf(scy), 0, ch - 1);
        const float dL0 = ldf(J.lc + (size_t)ncy * cw + ncx) - L0;
        const float sim0 = 1.0f / (1.0f + dL0 * dL0 * invSigma2);
        rescue = J.rescue * guideFade * phaseGate * phaseGate * (1.0f - sim0);
        if (rescue > 0.0f) {
            float kappa;
            if (!J.radial) {
                float mxX = 0, ssX = 0, mxY = 0, ssY = 0;
                for (int i = 0; i < ax.sup; ++i)
                    if (__ldg(amx + i) > 0) {
                        const float w = __ldg(wxp + i);
                        mxX = smax(mxX, fabsf(w));
                        ssX += w * w;
                    }
                for (int j = 0; j < ay.sup; ++j)
                    if (__ldg(amy + j) > 0) {
                        const float w = __ldg(wyp + j);
                        mxY = smax(mxY, fabsf(w));
                        ssY += w * w;
                    }
                kappa = (mxX * mxX * mxY * mxY) / (ssX * ssY + 1e-12f);
            } else {
                const float *base = radialWeightsAt(J.rad, ox, oy);
                float mx = 0, ss = 0;
                for (int j = 0; j < ay.sup; ++j) {
                    if (__ldg(amy + j) == 0) continue;
                    const float dyc = ((float)(ty0 + j) - scy) * J.invWyC;
                    for (int i = 0; i < ax.sup; ++i) {
                        if (__ldg(amx + i) == 0) continue;
                        const float dxc = ((float)(tx0 + i) - scx) * J.invWxC;
                        const float w = base ? ldf(base + (size_t)j * ax.sup + i)
                            : lutLookupDev(J.lut, J.lutN, sqrtf(dxc * dxc + dyc * dyc) * J.lutScale);
                        mx = smax(mx, fabsf(w));
                        ss += w * w;
                    }
                }
                kappa = (mx * mx) / (ss + 1e-12f);
            }
            rescue *= kappa * kappa;
        }
    }
    const float aniso = 1.0f + J.stretch * dir.coherence;
    const float invG2 = J.invGsigma2;
    const float invG2Par = invG2 / (aniso * aniso);

    // pass 2: sup x sup taps with w = sim * (wbase + rescue * bump)
    double accU = 0.0, accV = 0.0, wsum = 0.0, sumAbs = 0.0;
    const float *base = J.radial ? radialWeightsAt(J.rad, ox, oy) : nullptr;
    for (int j = 0; j < ay.sup; ++j) {
        if (__ldg(amy + j) == 0)
            continue;
        const size_t rowOff = (size_t)iclamp(ty0 + j, 0, ch - 1) * cw;
        const float wy = __ldg(wyp + j);
        const float dyf = (float)(ty0 + j) - scy;
        const float dy = dyf * J.rhF;
        const float dyc = dyf * J.invWyC;
        for (int i = 0; i < ax.sup; ++i) {
            if (__ldg(amx + i) == 0)
                continue;
            const size_t o = rowOff + iclamp(tx0 + i, 0, cw - 1);
            const float dxf = (float)(tx0 + i) - scx;
            float wx;
            if (base)
                wx = ldf(base + (size_t)j * ax.sup + i);
            else if (J.radial) {
                const float dxc = dxf * J.invWxC;
                wx = lutLookupDev(J.lut, J.lutN, sqrtf(dxc * dxc + dyc * dyc) * J.lutScale);
            } else
                wx = __ldg(wxp + i) * wy;
            const float dx = dxf * J.rwF;
            const float dL = ldf(J.lc + o) - L0;
            const float dp = dx * nx + dy * ny;
            const float dt = -dx * ny + dy * nx;
            const float simRaw = 1.0f / (1.0f + dL * dL * invSigma2);
            const float sim = 1.0f - guideFade * (1.0f - simRaw);
            const float bump = 1.0f / (1.0f + dp * dp * invG2 + dt * dt * invG2Par);
            const float w = sim * (wx + rescue * bump);
            const double wd = (double)w;
            accU = fma(wd, (double)ldf(J.U + o), accU);
            accV = fma(wd, (double)ldf(J.V + o), accV);
            wsum += wd;
            sumAbs += (double)fabsf(w);
        }
    }
    double valueU, valueV;
    if (wsum > 1e-6 && wsum >= 0.05 * sumAbs) {
        valueU = accU / wsum;
        valueV = accV / wsum;
    } else {
        valueU = bilinearAt(J.U, cw, ch, scx, scy);
        valueV = bilinearAt(J.V, cw, ch, scx, scy);
    }
    if (J.clampHull) {
        valueU = sclamp(valueU, (double)(hMinU - J.margin), (double)(hMaxU + J.margin));
        valueV = sclamp(valueV, (double)(hMinV - J.margin), (double)(hMaxV + J.margin));
    }
    g.u = valueU;
    g.v = valueV;
    g.L0 = L0;
    g.ssRamp = ssRamp;
    g.guideFade = guideFade;
    g.nx = nx;
    g.ny = ny;
    g.hasDir = hasDir;
    return g;
}

__device__ __forceinline__ bool pixelActive(const FrameJob &J, int ox, int oy) {
    if (!J.sparse)
        return true;
    const int mx = J.sameSize ? ox : min(J.sw - 1, (int)((long long)ox * J.sw / J.W));
    const int my = J.sameSize ? oy : min(J.sh - 1, (int)((long long)oy * J.sh / J.H));
    return J.mask[(size_t)my * J.sw + mx] != 0;
}

// Final sample of one output pixel: to the typed output plane when this
// stage is the last one touching it, else to the float planes.
__device__ __forceinline__ void emit(const FrameJob &J, int ox, int oy, float u, float v) {
    if (J.directOutput) {
        storeChroma(J, 1, ox, oy, u);
        storeChroma(J, 2, ox, oy, v);
    } else {
        const size_t o = (size_t)oy * J.W + ox;
        J.oU[o] = u;
        J.oV[o] = v;
    }
}

__global__ void __launch_bounds__(256)
k_recon(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int ox, oy;
    tile32x8(blockIdx.x - tileStart[f], J.W, ox, oy);
    if (ox >= J.W || oy >= J.H)
        return;
    if (!J.guided) {                                   // strength == 0: plain only
        float u, v;
        plainPixel(J, ox, oy, u, v);
        emit(J, ox, oy, u, v);
        return;
    }
    if (J.algo == 2) {
        const bool active = pixelActive(J, ox, oy);
        if (!active) {                                 // sparse: plain kernel suffices
            float u, v;
            plainPixel(J, ox, oy, u, v);
            emit(J, ox, oy, u, v);
            return;
        }
        const Guided g = guidedPixel(J, ox, oy);
        emit(J, ox, oy, (float)g.u, (float)g.v);
        return;
    }
    if (J.algo == 6) {                                 // plain base; detail later
        float u, v;
        plainPixel(J, ox, oy, u, v);
        emit(J, ox, oy, u, v);
        return;
    }
    // algo 4: plain base plus guided routing (recon.cpp:762-811)
    float baseU, baseV;
    plainPixel(J, ox, oy, baseU, baseV);
    const size_t o = (size_t)oy * J.W + ox;
    if (!pixelActive(J, ox, oy)) {
        if (J.outKind == kF32) {
            J.oU[o] = baseU;
            J.oV[o] = baseV;
        } else {
            emit(J, ox, oy, baseU, baseV);
        }
        return;
    }
    const Guided g = guidedPixel(J, ox, oy);
    const float diag = g.hasDir ? smin(1.0f, 2.0f * fabsf(g.nx * g.ny)) : 0.0f;
    const float hedgy = (1.0f - g.ssRamp) * g.guideFade;
    const float sel = J.strength4;
    const float w2 = hedgy * (1.0f - diag) * sel;
    const float w3 = hedgy * diag * sel;
    if (J.outKind != kF32) {
        // integer output: single-expression fused selector
        double valueU, valueV;
        if (w2 >= 1e-4f || w3 >= 1e-4f) {
            const int cx = __ldg(J.ax.cbI0 + ox), cy = __ldg(J.ay.cbI0 + oy);
            const float cxf = __ldg(J.ax.cbF + ox), cyf = __ldg(J.ay.cbF + oy);
            const size_t plane = (size_t)J.cw * J.ch;
            const float au = bilinearFast(J.lgf + 0 * plane, J.cw, J.ch, cx, cxf, cy, cyf);
            const float bu = bilinearFast(J.lgf + 1 * plane, J.cw, J.ch, cx, cxf, cy, cyf);
            const float cu = bilinearFast(J.lgf + 2 * plane, J.cw, J.ch, cx, cxf, cy, cyf);
            const float av = bilinearFast(J.lgf + 3 * plane, J.cw, J.ch, cx, cxf, cy, cyf);
            const float bv = bilinearFast(J.lgf + 4 * plane, J.cw, J.ch, cx, cxf, cy, cyf);
            const float cv = bilinearFast(J.lgf + 5 * plane, J.cw, J.ch, cx, cxf, cy, cyf);
            valueU = baseU + w2 * ((float)g.u - baseU) + w3 * cu * (au * g.L0 + bu - baseU);
            valueV = baseV + w2 * ((float)g.v - baseV) + w3 * cv * (av * g.L0 + bv - baseV);
        } else {
            valueU = baseU;
            valueV = baseV;
        }
        emit(J, ox, oy, (float)valueU, (float)valueV);
        return;
    }
    // float output: routing metadata; blended after the ROI-limited LGF
    J.oU[o] = baseU;
    J.oV[o] = baseV;
    const bool compressed = J.sparse &&
        (unsigned long long)J.counters[kCntActiveOutput] * 2ull < (unsigned long long)J.W * J.H;
    if (compressed) {
        if (w2 < 1e-4f && w3 < 1e-4f) {
            J.gU[o] = 0.0f;
            J.gV[o] = 0.0f;
            J.selW3[o] = 0.0f;
        } else {
            J.gU[o] = hedgy * (1.0f - diag) * ((float)g.u - baseU);
            J.gV[o] = hedgy * (1.0f - diag) * ((float)g.v - baseV);
            J.selW3[o] = hedgy * diag;
        }
    } else {
        J.gU[o] = (float)g.u;
        J.gV[o] = (float)g.v;
        J.selW2[o] = hedgy * (1.0f - diag);
        J.selW3[o] = hedgy * diag;
    }
}

// Float output planes -> typed output (output conversion stage).
__global__ void k_store_chroma(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart,
                               int njobs) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int ox, oy;
    tile32x8(blockIdx.x - tileStart[f], J.W, ox, oy);
    if (ox >= J.W || oy >= J.H)
        return;
    const size_t o = (size_t)oy * J.W + ox;
    storeChroma(J, 1, ox, oy, J.oU[o]);
    storeChroma(J, 2, ox, oy, J.oV[o]);
}

// ---------------------------------------------------------------------------
// Luma resize (output size differs): separable resampleH then resampleV
// (double accumulation, clamped taps), or the 2D jinc resampleRadial.
// ---------------------------------------------------------------------------
__global__ void k_luma_h(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart,
                         int njobs) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int x, y;
    tile32x8(blockIdx.x - tileStart[f], J.W, x, y);
    if (x >= J.W || y >= J.sh)
        return;
    const WeightView &t = J.lumaH;
    const int s = __ldg(t.start + x);
    const float *wp = t.w + (size_t)x * t.sup;
    const float *row = J.Y + (size_t)y * J.sw;
    double acc = 0.0;
    for (int j = 0; j < t.sup; ++j)
        acc = fma((double)__ldg(wp + j), (double)ldf(row + iclamp(s + j, 0, J.sw - 1)), acc);
    J.lumaTmp[(size_t)y * J.W + x] = (float)acc;
}

__global__ void k_luma_v(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart,
                         int njobs) {
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
                  (double)ldf(J.lumaTmp + (size_t)iclamp(s + j, 0, J.sh - 1) * J.W + x), acc);
    storeLuma(J, x, y, (float)acc);
}

__global__ void k_luma_radial(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart,
                              int njobs) {
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
        const float *row = J.Y + (size_t)ty * J.sw;
        for (int i = 0; i < sup; ++i) {
            const int tx = iclamp(x0 + i, 0, J.sw - 1);
            const float dx = (float)((x0 + i - cx) * invW);
            const float w = lutLookupDev(J.lut, J.lutN, sqrtf(dx * dx + dy * dy) * J.lutScale);
            acc = fma((double)w, (double)ldf(row + tx), acc);
            wsum += (double)w;
        }
    }
    storeLuma(J, ox, oy, (float)(wsum > 1e-6 ? acc / wsum : 0.0));
}

} // namespace lgcr_b200
