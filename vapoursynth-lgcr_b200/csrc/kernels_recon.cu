// Chroma reconstruction stages.
//   k_hpass   horizontal pass of the separable kernels: per (output column,
//             chroma row) the plain horizontal sums of U, V and the window
//             extrema of U, V, lc over the active taps (the reference's
//             ring rows, plainChromaSeparable src/recon.cpp:1178-1271)
//   k_plain   plain base per output pixel: vertical pass over the table
//             (separable, src/recon.cpp:1281-1437), bilinear
//             (src/recon.cpp:1031-1149) or radial (src/recon.cpp:828-1029);
//             writes the final sample of pixels the guided pass skips and,
//             for the pixels it lists, folds their guided windows' extrema
//   k_guided  reconstructChromaImpl (scalar, src/recon.cpp:14-819) for the
//             active pixels of every frame in the launch: a persistent grid
//             walks the frames' compacted work lists (no divergence between
//             plain and guided pixels). Pass 1 (window luma range and chroma
//             hull) reads the extrema k_plain folded (or the horizontal
//             table); pass 2 is specialized on the tap support so per-column
//             terms stay in registers.
//   luma resize       resampleH/V, resampleRadial src/kernels.cpp:171-334
//   output store      floatToPlane src/lgcr.h:997-1013
// FP64 accumulators stay FP64 (B200 issues FP64 at half the FP32 rate); a
// product of two floats is exact in double, so fma(w, u, acc) rounds exactly
// like the reference's acc += double(w) * u.
#include "kernels.cuh"
#include "temporal.cuh"
#include "plain.cuh"

namespace lgcr_b200 {

// ---------------------------------------------------------------------------
// horizontal table: hu hv mnU mxU | mnV mxV mnL mxL per (output column,
// chroma row) over the column's active taps
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t maskBits(const uint8_t *am, int n) {
    uint32_t m = 0;
    for (int i = 0; i < n; ++i)
        m |= (__ldg(am + i) != 0 ? 1u : 0u) << i;
    return m;
}

// Tap data of one output column (start, activity bits, FP64 weights), loaded
// once and reused for every chroma row the column is evaluated on.
template <int SUP>
struct HColumn {
    int tx0;
    uint32_t active;
    double w[SUP];
    __device__ __forceinline__ void load(const AxisView &ax, int ox) {
        tx0 = __ldg(ax.start + ox);
        active = maskBits(ax.am + (size_t)ox * SUP, SUP);
#pragma unroll
        for (int i = 0; i < SUP; ++i)
            w[i] = __ldg(ax.wd + (size_t)ox * SUP + i);
    }
};

// LUMA: also the extrema of lc (read only by the guided pass: the folded
// window extrema or the horizontal table).
template <int SUP, bool NOCLAMP, bool LUMA = true>
__device__ __forceinline__ void hEntry(const FrameJob &J, const HColumn<SUP> &col, int sy, float4 &ea,
                                       float4 &eb) {
    const int cw = J.cw;
    const size_t row = (size_t)sy * cw;
    const double2 *uv = reinterpret_cast<const double2 *>(J.uvd) + row;
    const float *lrow = (LUMA && J.lc) ? J.lc + row : nullptr;
    double hU = 0.0, hV = 0.0;
    // extrema of the float samples: the doubles hold them exactly, so they
    // narrow back without a second load
    float mnU = 1e30f, mxU = -1e30f, mnV = 1e30f, mxV = -1e30f;
    float mnL = 1e30f, mxL = -1e30f;
#pragma unroll
    for (int i = 0; i < SUP; ++i) {
        if (!((col.active >> i) & 1u))
            continue;
        const int x = NOCLAMP ? col.tx0 + i : iclamp(col.tx0 + i, 0, cw - 1);
        const double2 p = __ldg(uv + x);
        const double w = col.w[i];
        hU = fma(w, p.x, hU);
        hV = fma(w, p.y, hV);
        const float u = (float)p.x, v = (float)p.y;
        mnU = runMin(mnU, u); mxU = runMax(mxU, u);
        mnV = runMin(mnV, v); mxV = runMax(mxV, v);
        if (LUMA && lrow) {
            const float l = ldf(lrow + x);
            mnL = runMin(mnL, l); mxL = runMax(mxL, l);
        }
    }
    ea = make_float4((float)hU, (float)hV, mnU, mxU);
    eb = make_float4(mnV, mxV, mnL, mxL);
}

// Any support (activity read per tap).
__device__ __forceinline__ void hEntryGeneric(const FrameJob &J, int ox, int sy, float4 &ea, float4 &eb) {
    const AxisView &ax = J.ax;
    const int n = ax.sup;
    const int cw = J.cw;
    const int tx0 = __ldg(ax.start + ox);
    const double *wx = ax.wd + (size_t)ox * ax.sup;
    const uint8_t *amx = ax.am + (size_t)ox * ax.sup;
    const double2 *uv = reinterpret_cast<const double2 *>(J.uvd) + (size_t)sy * cw;
    const float *lrow = J.lc ? J.lc + (size_t)sy * cw : nullptr;
    double hU = 0.0, hV = 0.0;
    double mnU = 1e30f, mxU = -1e30f, mnV = 1e30f, mxV = -1e30f;
    float mnL = 1e30f, mxL = -1e30f;
    for (int i = 0; i < n; ++i) {
        if (__ldg(amx + i) == 0)
            continue;
        const int x = J.noClampX ? tx0 + i : iclamp(tx0 + i, 0, cw - 1);
        const double2 p = __ldg(uv + x);
        const double w = __ldg(wx + i);
        hU = fma(w, p.x, hU);
        hV = fma(w, p.y, hV);
        mnU = runMin(mnU, p.x); mxU = runMax(mxU, p.x);
        mnV = runMin(mnV, p.y); mxV = runMax(mxV, p.y);
        if (lrow) {
            const float l = ldf(lrow + x);
            mnL = runMin(mnL, l); mxL = runMax(mxL, l);
        }
    }
    ea = make_float4((float)hU, (float)hV, (float)mnU, (float)mxU);
    eb = make_float4((float)mnV, (float)mxV, mnL, mxL);
}

__device__ __forceinline__ void storeEntry(const FrameJob &J, int ox, int sy, const float4 &ea,
                                           const float4 &eb) {
    float4 *o = reinterpret_cast<float4 *>(J.hTab + ((size_t)sy * J.W + ox) * 8);
    o[0] = ea;
    o[1] = eb;
}

// Standalone horizontal pass (frames whose plain blocks cannot stage their
// rows in shared memory).
__global__ void __launch_bounds__(256)
k_hpass(LGCR_STAGE_ARGS) {
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    int ox, sy;
    tile32x8(blockIdx.x - tileStart[f], J.W, ox, sy);
    if (ox >= J.W || sy >= J.ch)
        return;
    float4 a, b;
    switch (J.ax.sup) {
    case 4: { HColumn<4> c; c.load(J.ax, ox); if (J.noClampX) hEntry<4, true>(J, c, sy, a, b); else hEntry<4, false>(J, c, sy, a, b); break; }
    case 6: { HColumn<6> c; c.load(J.ax, ox); if (J.noClampX) hEntry<6, true>(J, c, sy, a, b); else hEntry<6, false>(J, c, sy, a, b); break; }
    case 8: { HColumn<8> c; c.load(J.ax, ox); if (J.noClampX) hEntry<8, true>(J, c, sy, a, b); else hEntry<8, false>(J, c, sy, a, b); break; }
    default: hEntryGeneric(J, ox, sy, a, b); break;
    }
    storeEntry(J, ox, sy, a, b);
}

// Plain separable value from the horizontal table (vertical pass).
template <int SUP>
__device__ __forceinline__ void plainFromTableT(const FrameJob &J, int ox, int oy, float &outU,
                                                float &outV) {
    const AxisView &ax = J.ax, &ay = J.ay;
    const int n = SUP > 0 ? SUP : ay.sup;
    const int ty0 = __ldg(ay.start + oy);
    const double *wy = ay.wd + (size_t)oy * ay.sup;
    const uint8_t *amy = ay.am + (size_t)oy * ay.sup;
    double vU = 0.0, vV = 0.0;
    float mnU = 1e30f, mxU = -1e30f, mnV = 1e30f, mxV = -1e30f;
#pragma unroll
    for (int j = 0; j < n; ++j) {
        if (__ldg(amy + j) == 0)
            continue;
        const int sy = J.noClampY ? ty0 + j : iclamp(ty0 + j, 0, J.ch - 1);
        const float4 *h = reinterpret_cast<const float4 *>(J.hTab + ((size_t)sy * J.W + ox) * 8);
        const float4 a = __ldg(h), b = __ldg(h + 1);
        const double w = __ldg(wy + j);
        vU = fma(w, (double)a.x, vU);
        vV = fma(w, (double)a.y, vV);
        mnU = runMin(mnU, a.z); mxU = runMax(mxU, a.w);
        mnV = runMin(mnV, b.x); mxV = runMax(mxV, b.y);
    }
    const double ws = (double)__ldg(ax.wsum + ox) * (double)__ldg(ay.wsum + oy);
    const double wa = (double)__ldg(ax.wabs + ox) * (double)__ldg(ay.wabs + oy);
    if (ws > 1e-6 && ws >= 0.05 * wa) {
        vU /= ws;
        vV /= ws;
    } else {
        const float px = __ldg(ax.pos + ox), py = __ldg(ay.pos + oy);
        vU = bilinearAt(J.U, J.cw, J.ch, px, py);
        vV = bilinearAt(J.V, J.cw, J.ch, px, py);
    }
    if (J.clampHull) {
        vU = sclamp(vU, (double)(mnU - J.margin), (double)(mxU + J.margin));
        vV = sclamp(vV, (double)(mnV - J.margin), (double)(mxV + J.margin));
    }
    outU = (float)vU;
    outV = (float)vV;
}

__device__ __forceinline__ void plainFromTable(const FrameJob &J, int ox, int oy, float &u, float &v) {
    switch (J.ay.sup) {
    case 4: plainFromTableT<4>(J, ox, oy, u, v); break;
    case 6: plainFromTableT<6>(J, ox, oy, u, v); break;
    case 8: plainFromTableT<8>(J, ox, oy, u, v); break;
    default: plainFromTableT<0>(J, ox, oy, u, v); break;
    }
}

__device__ __forceinline__ void plainPixel(const FrameJob &J, int ox, int oy, float &u, float &v) {
    if (!J.radial && J.kernel != 0 && J.hTab)
        plainFromTable(J, ox, oy, u, v);
    else
        plainAt(chromaPlainCtx(J), ox, oy, u, v);
}

__device__ __forceinline__ bool pixelActive(const FrameJob &J, int ox, int oy) {
    if (!J.sparse)
        return true;
    const int mx = J.sameSize ? ox : min(J.sw - 1, (int)((long long)ox * J.sw / J.W));
    const int my = J.sameSize ? oy : min(J.sh - 1, (int)((long long)oy * J.sh / J.H));
    return maskAt(J, mx, my) != 0;
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

// Vertical pass over table rows staged in shared memory: same arithmetic and
// order as plainFromTableT, rows indexed relative to the staged block. The
// horizontal sums are staged as the float-rounded ring value and widened to
// double (exact) where the reference multiplies them in double.
template <int SUP>
__device__ __forceinline__ void plainFromStaged(const FrameJob &J, const float2 (*sHV)[32],
                                                const float4 (*sE)[32], int syLo, int lx, int ox,
                                                int oy, float &outU, float &outV) {
    const AxisView &ax = J.ax, &ay = J.ay;
    const int n = SUP > 0 ? SUP : ay.sup;
    const int ty0 = __ldg(ay.start + oy);
    const double *wy = ay.wd + (size_t)oy * ay.sup;
    const uint8_t *amy = ay.am + (size_t)oy * ay.sup;
    double vU = 0.0, vV = 0.0;
    float mnU = 1e30f, mxU = -1e30f, mnV = 1e30f, mxV = -1e30f;
#pragma unroll
    for (int j = 0; j < n; ++j) {
        if (__ldg(amy + j) == 0)
            continue;
        const int r = (J.noClampY ? ty0 + j : iclamp(ty0 + j, 0, J.ch - 1)) - syLo;
        const float2 h = sHV[r][lx];
        const float4 e = sE[r][lx];
        const double w = __ldg(wy + j);
        vU = fma(w, (double)h.x, vU);
        vV = fma(w, (double)h.y, vV);
        mnU = runMin(mnU, e.x); mxU = runMax(mxU, e.y);
        mnV = runMin(mnV, e.z); mxV = runMax(mxV, e.w);
    }
    const double ws = (double)__ldg(ax.wsum + ox) * (double)__ldg(ay.wsum + oy);
    const double wa = (double)__ldg(ax.wabs + ox) * (double)__ldg(ay.wabs + oy);
    if (ws > 1e-6 && ws >= 0.05 * wa) {
        vU /= ws;
        vV /= ws;
    } else {
        const float px = __ldg(ax.pos + ox), py = __ldg(ay.pos + oy);
        vU = bilinearAt(J.U, J.cw, J.ch, px, py);
        vV = bilinearAt(J.V, J.cw, J.ch, px, py);
    }
    if (J.clampHull) {
        vU = sclamp(vU, (double)(mnU - J.margin), (double)(mxU + J.margin));
        vV = sclamp(vV, (double)(mnV - J.margin), (double)(mxV + J.margin));
    }
    outU = (float)vU;
    outV = (float)vV;
}

// Position of the n-th (0-based) set bit of m (n < popc(m)): the largest p
// with fewer than n + 1 set bits below p.
__device__ __forceinline__ int nthSetBit(uint32_t m, int n) {
    int pos = 0;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1)
        if (__popc(m & ((1u << (pos + s)) - 1u)) <= n)
            pos += s;
    return pos;
}

// Per-row vertical tap data of one k_plain block, staged once for the
// block's output rows (at most kPlainRows; supports up to 8 taps).
struct PlainRows {
    double w[kPlainRows][8];
    int ty0[kPlainRows];
    uint32_t act[kPlainRows];
    float wsum[kPlainRows], wabs[kPlainRows], pos[kPlainRows];
    uint32_t maskWord[kPlainRows];     // active-pixel bits of the block's 32 columns
};

// The same vertical pass with the row data from PlainRows and the column
// data (wsX, waX, posX) held in registers.
template <int SUP, bool NOCLAMP>
__device__ __forceinline__ void plainFromRows(const FrameJob &J, const float2 (*sHV)[32],
                                              const float4 (*sE)[32], const PlainRows &R, int k,
                                              int syLo, int lx, float wsX, float waX, float posX,
                                              float &outU, float &outV) {
    const int ty0 = R.ty0[k];
    const uint32_t act = R.act[k];
    double vU = 0.0, vV = 0.0;
    float mnU = 1e30f, mxU = -1e30f, mnV = 1e30f, mxV = -1e30f;
#pragma unroll
    for (int j = 0; j < SUP; ++j) {
        if (!((act >> j) & 1u))
            continue;
        const int r = (NOCLAMP ? ty0 + j : iclamp(ty0 + j, 0, J.ch - 1)) - syLo;
        const float2 h = sHV[r][lx];
        const float4 e = sE[r][lx];
        const double w = R.w[k][j];
        vU = fma(w, (double)h.x, vU);
        vV = fma(w, (double)h.y, vV);
        mnU = runMin(mnU, e.x); mxU = runMax(mxU, e.y);
        mnV = runMin(mnV, e.z); mxV = runMax(mxV, e.w);
    }
    const double ws = (double)wsX * (double)R.wsum[k];
    const double wa = (double)waX * (double)R.wabs[k];
    if (ws > 1e-6 && ws >= 0.05 * wa) {
        vU /= ws;
        vV /= ws;
    } else {
        vU = bilinearAt(J.U, J.cw, J.ch, posX, R.pos[k]);
        vV = bilinearAt(J.V, J.cw, J.ch, posX, R.pos[k]);
    }
    if (J.clampHull) {
        vU = sclamp(vU, (double)(mnU - J.margin), (double)(mxU + J.margin));
        vV = sclamp(vV, (double)(mnV - J.margin), (double)(mxV + J.margin));
    }
    outU = (float)vU;
    outV = (float)vV;
}

// Shared-memory rows of one k_plain block: float-rounded horizontal sums
// (widened to double where the vertical pass multiplies them), chroma hull and (frames whose guided pass reads the folded extrema) luma
// extrema of each staged (chroma row, output column).
struct PlainStage {
    float2 (*hv)[32];
    float4 (*e)[32];
    float2 (*l)[32];
};

// Horizontal entries of the rows [syLo, syLo + nRows) for output column ox
// into shared memory; table rows this block owns (sy < syOwnEnd) also go to
// the frame's horizontal table for the guided pass. Two rows per step keep
// both rows' loads in flight together.
__device__ __forceinline__ void putEntry(const FrameJob &J, int ox, int lx, int r, int sy, const float4 &a,
                                         const float4 &b, int syOwnEnd, bool writeTable,
                                         const PlainStage &s) {
    s.hv[r][lx] = make_float2(a.x, a.y);
    s.e[r][lx] = make_float4(a.z, a.w, b.x, b.y);
    if (J.wLum)
        s.l[r][lx] = make_float2(b.z, b.w);
    if (writeTable && sy < syOwnEnd)
        storeEntry(J, ox, sy, a, b);
}

template <int SUP, bool NOCLAMP, bool LUMA>
__device__ __forceinline__ void stageRowsT(const FrameJob &J, const HColumn<SUP> &col, int ox, int lx,
                                           int syLo, int nRows, int syOwnEnd, bool writeTable,
                                           const PlainStage &s) {
    const int step = blockDim.y;
    int r = threadIdx.y;
    for (; r + step < nRows; r += 2 * step) {
        float4 a0, b0, a1, b1;
        hEntry<SUP, NOCLAMP, LUMA>(J, col, syLo + r, a0, b0);
        hEntry<SUP, NOCLAMP, LUMA>(J, col, syLo + r + step, a1, b1);
        putEntry(J, ox, lx, r, syLo + r, a0, b0, syOwnEnd, writeTable, s);
        putEntry(J, ox, lx, r + step, syLo + r + step, a1, b1, syOwnEnd, writeTable, s);
    }
    if (r < nRows) {
        float4 a, b;
        hEntry<SUP, NOCLAMP, LUMA>(J, col, syLo + r, a, b);
        putEntry(J, ox, lx, r, syLo + r, a, b, syOwnEnd, writeTable, s);
    }
}

template <int SUP>
__device__ __forceinline__ void stageRows(const FrameJob &J, int ox, int lx, int syLo, int nRows,
                                          int syOwnEnd, bool writeTable, const PlainStage &s) {
    HColumn<SUP> col;
    col.load(J.ax, ox);
    // the luma extrema only feed the guided pass (folded planes or the table)
    if (J.wLum || writeTable) {
        if (J.noClampX)
            stageRowsT<SUP, true, true>(J, col, ox, lx, syLo, nRows, syOwnEnd, writeTable, s);
        else
            stageRowsT<SUP, false, true>(J, col, ox, lx, syLo, nRows, syOwnEnd, writeTable, s);
    } else {
        if (J.noClampX)
            stageRowsT<SUP, true, false>(J, col, ox, lx, syLo, nRows, syOwnEnd, writeTable, s);
        else
            stageRowsT<SUP, false, false>(J, col, ox, lx, syLo, nRows, syOwnEnd, writeTable, s);
    }
}

__device__ __forceinline__ void stageRowsGeneric(const FrameJob &J, int ox, int lx, int syLo, int nRows,
                                                 int syOwnEnd, bool writeTable, const PlainStage &s) {
    for (int r = threadIdx.y; r < nRows; r += blockDim.y) {
        float4 a, b;
        hEntryGeneric(J, ox, syLo + r, a, b);
        putEntry(J, ox, lx, r, syLo + r, a, b, syOwnEnd, writeTable, s);
    }
}

// Extrema of a listed pixel's guided window (pass 1 of reconstructChromaImpl,
// src/recon.cpp:258-367: the chroma hull and the luma range over the active
// taps) folded from the staged rows in the same row order as the guided
// pass's own fold, to the frame's extrema planes.
template <int SUP, bool NOCLAMP>
__device__ __forceinline__ void extremaFromRows(const FrameJob &J, const float4 (*sE)[32],
                                                const float2 (*sL)[32], const PlainRows &R, int k,
                                                int syLo, int lx, size_t o) {
    const int ty0 = R.ty0[k];
    const uint32_t act = R.act[k];
    float mnU = 1e30f, mxU = -1e30f, mnV = 1e30f, mxV = -1e30f, mnL = 1e30f, mxL = -1e30f;
#pragma unroll
    for (int j = 0; j < SUP; ++j) {
        if (!((act >> j) & 1u))
            continue;
        const int r = (NOCLAMP ? ty0 + j : iclamp(ty0 + j, 0, J.ch - 1)) - syLo;
        const float4 e = sE[r][lx];
        const float2 l = sL[r][lx];
        mnU = runMin(mnU, e.x); mxU = runMax(mxU, e.y);
        mnV = runMin(mnV, e.z); mxV = runMax(mxV, e.w);
        mnL = runMin(mnL, l.x); mxL = runMax(mxL, l.y);
    }
    J.wHull[o] = make_float4(mnU, mxU, mnV, mxV);
    J.wLum[o] = make_float2(mnL, mxL);
}

// Plain stage: every pixel the guided pass does not finalize. A block covers
// 32 output columns x J.plainRows output rows. For the separable kernels it
// needs the horizontal entries of the chroma rows its windows touch:
//  * fused frames (every block's rows fit in shared memory) compute them
//    here from the chroma planes (the reference's ring rows), and write the
//    rows the block owns to the horizontal table when the guided pass reads
//    it (chroma row sy is owned by the last block whose rows start at or
//    before sy, so every row some window reads is written exactly once);
//  * other frames stage rows of the table written by k_hpass, or read the
//    table directly when the rows do not fit (strong vertical downscale).
// The vertical pass then runs from shared memory, with the per-row tap data
// and active-pixel bits staged once per block for supports up to 8. Pixels
// the guided pass lists get their window extrema folded instead (frames
// with extrema planes), and each warp compacts its remaining plain pixels
// across its rows so full warps evaluate them.
template <bool EARLY>
__device__ __forceinline__ void plainStage(const FrameJob *__restrict__ jobs,
                                           const int *__restrict__ tileStart, int njobs) {
    extern __shared__ __align__(16) unsigned char plainRowsSmem[];
    float2 (*sHV)[32] = reinterpret_cast<float2 (*)[32]>(plainRowsSmem);
    float4 (*sE)[32] = reinterpret_cast<float4 (*)[32]>(      // mnU mxU mnV mxV
        plainRowsSmem + size_t(kPlainStagedRows) * 32 * 8);
    float2 (*sL)[32] = reinterpret_cast<float2 (*)[32]>(      // mnL mxL
        plainRowsSmem + size_t(kPlainStagedRows) * 32 * 24);
    __shared__ PlainRows R;
    __shared__ FrameJob sJob;
    __shared__ uint32_t sRowBits[8][kPlainRows / 8];   // per warp: plain pixels of its rows
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    stageJob(jobs, f, sJob);
    const FrameJob &J = sJob;
    const int tile = blockIdx.x - tileStart[f];
    const int tilesX = (J.W + 31) >> 5;
    const int colBase = (tile % tilesX) * 32;
    const int oy0 = (tile / tilesX) * J.plainRows;
    const int rowsHere = min(J.plainRows, J.H - oy0);
    const int lx = threadIdx.x;
    const int ox = colBase + lx;
    const int tid = threadIdx.y * 32 + lx;
    const bool separable = !J.radial && J.kernel != 0;
    const bool fused = J.plainFused && (separable || J.listed);
    const bool table = separable && (J.hTab || fused);
    const bool floatSelector = J.guided && J.algo == 4 && J.outKind == kF32;
    const bool skipListed = J.listed && (!floatSelector || radialPlainFused(J));
    // every output pixel listed (the trust mask covers the frame) and no
    // table or extrema for the guided pass to produce here: the guided pass
    // writes every pixel and nothing here is needed (EARLY instance only:
    // compiled into the common one, the test costs the separable frames'
    // plain pass 5 % through its register allocation)
    if (EARLY && skipListed && !J.hTab && !J.wHull && !J.finalInTransfer &&
        J.counters[kCntActiveOutput] >= (unsigned long long)J.W * J.H)
        return;
    int syLo = 0, nRows = 0;
    if (table || fused) {
        const int oyLast = oy0 + rowsHere - 1;
        syLo = iclamp(__ldg(J.ay.start + oy0), 0, J.ch - 1);
        const int syHi = iclamp(__ldg(J.ay.start + oyLast) + J.ay.sup - 1, 0, J.ch - 1);
        nRows = syHi - syLo + 1;
    }
    const bool staged = (table || fused) && nRows <= kPlainStagedRows;
    const int sup = J.ay.sup;
    const bool rowTables = table && staged && sup <= 8;
    if (rowTables) {
        for (int i = tid; i < rowsHere * sup; i += 256) {
            const int k = i / sup, j = i - k * sup;
            R.w[k][j] = __ldg(J.ay.wd + (size_t)(oy0 + k) * sup + j);
        }
        if (tid < rowsHere) {
            const int oy = oy0 + tid;
            R.ty0[tid] = __ldg(J.ay.start + oy);
            R.act[tid] = maskBits(J.ay.am + (size_t)oy * sup, sup);
            R.wsum[tid] = __ldg(J.ay.wsum + oy);
            R.wabs[tid] = __ldg(J.ay.wabs + oy);
            R.pos[tid] = __ldg(J.ay.pos + oy);
        }
    }
    // active-pixel bits: listed pixels are skipped here (after folding their
    // guided windows' extrema); algo 6 pixels the detail transfer leaves
    // alone are stored final here
    const bool foldExtrema = J.wHull != nullptr;    // implies fused row tables
    const bool needAct = skipListed || J.finalInTransfer || foldExtrema;
    const bool maskWords = needAct && J.sparse && J.sameSize;
    if (maskWords && tid < rowsHere)
        R.maskWord[tid] = __ldg(J.mask + (size_t)(oy0 + tid) * J.maskWords + (colBase >> 5));
    if (fused) {
        // rows from the next block's first row on belong to the next block
        const int syOwnEnd = (oy0 + J.plainRows < J.H)
            ? iclamp(__ldg(J.ay.start + oy0 + J.plainRows), 0, J.ch - 1) : J.ch;
        const bool writeTable = J.listed && J.hTab;
        const PlainStage s{sHV, sE, sL};
        if (ox < J.W) {
            switch (J.ax.sup) {
            case 4: stageRows<4>(J, ox, lx, syLo, nRows, syOwnEnd, writeTable, s); break;
            case 6: stageRows<6>(J, ox, lx, syLo, nRows, syOwnEnd, writeTable, s); break;
            case 8: stageRows<8>(J, ox, lx, syLo, nRows, syOwnEnd, writeTable, s); break;
            default: stageRowsGeneric(J, ox, lx, syLo, nRows, syOwnEnd, writeTable, s); break;
            }
        }
    } else if (staged && ox < J.W) {
        for (int r = threadIdx.y; r < nRows; r += blockDim.y) {
            const float4 *h =
                reinterpret_cast<const float4 *>(J.hTab + ((size_t)(syLo + r) * J.W + ox) * 8);
            const float4 a = __ldg(h), b = __ldg(h + 1);
            sHV[r][lx] = make_float2(a.x, a.y);
            sE[r][lx] = make_float4(a.z, a.w, b.x, b.y);
        }
    }
    __syncthreads();
    const bool colValid = ox < J.W;
    float wsX = 0.0f, waX = 0.0f, posX = 0.0f;
    if (rowTables && colValid) {
        wsX = __ldg(J.ax.wsum + ox);
        waX = __ldg(J.ax.wabs + ox);
        posX = __ldg(J.ax.pos + ox);
    }
    if (skipListed && rowTables) {
        // Listed pixels only fold extrema here; the warp's plain pixels over
        // its rows (threadIdx.y + 8m) are compacted so full warps evaluate them.
        uint32_t *rowBits = sRowBits[threadIdx.y];
        int total = 0;
        for (int m = 0; m < kPlainRows / 8; ++m) {
            const int k = threadIdx.y + 8 * m;
            bool plainPx = false;
            if (k < rowsHere && colValid) {
                const int oy = oy0 + k;
                const bool act = maskWords ? ((R.maskWord[k] >> lx) & 1u) != 0 : pixelActive(J, ox, oy);
                if (act && foldExtrema) {
                    const size_t o = (size_t)oy * J.W + ox;
                    if (J.noClampY) {
                        switch (sup) {
                        case 4: extremaFromRows<4, true>(J, sE, sL, R, k, syLo, lx, o); break;
                        case 6: extremaFromRows<6, true>(J, sE, sL, R, k, syLo, lx, o); break;
                        default: extremaFromRows<8, true>(J, sE, sL, R, k, syLo, lx, o); break;
                        }
                    } else {
                        switch (sup) {
                        case 4: extremaFromRows<4, false>(J, sE, sL, R, k, syLo, lx, o); break;
                        case 6: extremaFromRows<6, false>(J, sE, sL, R, k, syLo, lx, o); break;
                        default: extremaFromRows<8, false>(J, sE, sL, R, k, syLo, lx, o); break;
                        }
                    }
                }
                plainPx = !act;
            }
            const uint32_t b = __ballot_sync(0xffffffffu, plainPx);
            if (lx == 0)
                rowBits[m] = b;
            total += __popc(b);
        }
        __syncwarp();
        for (int base = 0; base < total; base += 32) {
            const int j = base + lx;
            int m = 0, col = 0, before = 0;
            if (j < total) {
                uint32_t b = rowBits[0];
                while (before + __popc(b) <= j) {
                    before += __popc(b);
                    b = rowBits[++m];
                }
                col = nthSetBit(b, j - before);
            }
            const float wsC = __shfl_sync(0xffffffffu, wsX, col);
            const float waC = __shfl_sync(0xffffffffu, waX, col);
            const float posC = __shfl_sync(0xffffffffu, posX, col);
            if (j < total) {
                const int k = threadIdx.y + 8 * m;
                float u, v;
                if (J.noClampY) {
                    switch (sup) {
                    case 4: plainFromRows<4, true>(J, sHV, sE, R, k, syLo, col, wsC, waC, posC, u, v); break;
                    case 6: plainFromRows<6, true>(J, sHV, sE, R, k, syLo, col, wsC, waC, posC, u, v); break;
                    default: plainFromRows<8, true>(J, sHV, sE, R, k, syLo, col, wsC, waC, posC, u, v); break;
                    }
                } else {
                    switch (sup) {
                    case 4: plainFromRows<4, false>(J, sHV, sE, R, k, syLo, col, wsC, waC, posC, u, v); break;
                    case 6: plainFromRows<6, false>(J, sHV, sE, R, k, syLo, col, wsC, waC, posC, u, v); break;
                    default: plainFromRows<8, false>(J, sHV, sE, R, k, syLo, col, wsC, waC, posC, u, v); break;
                    }
                }
                emit(J, colBase + col, oy0 + k, u, v);
            }
        }
        return;
    }
    if (!colValid)
        return;
    for (int k = threadIdx.y; k < rowsHere; k += blockDim.y) {
        const int oy = oy0 + k;
        // listed pixels of algo 2 and integer algo 4 are written by k_guided
        bool act = false;
        if (needAct) {
            act = maskWords ? ((R.maskWord[k] >> lx) & 1u) != 0 : pixelActive(J, ox, oy);
            if (act && foldExtrema) {
                const size_t o = (size_t)oy * J.W + ox;
                if (J.noClampY) {
                    switch (sup) {
                    case 4: extremaFromRows<4, true>(J, sE, sL, R, k, syLo, lx, o); break;
                    case 6: extremaFromRows<6, true>(J, sE, sL, R, k, syLo, lx, o); break;
                    default: extremaFromRows<8, true>(J, sE, sL, R, k, syLo, lx, o); break;
                    }
                } else {
                    switch (sup) {
                    case 4: extremaFromRows<4, false>(J, sE, sL, R, k, syLo, lx, o); break;
                    case 6: extremaFromRows<6, false>(J, sE, sL, R, k, syLo, lx, o); break;
                    default: extremaFromRows<8, false>(J, sE, sL, R, k, syLo, lx, o); break;
                    }
                }
            }
            if (act && skipListed)
                continue;
        }
        float u, v;
        if (rowTables) {
            if (J.noClampY) {
                switch (sup) {
                case 4: plainFromRows<4, true>(J, sHV, sE, R, k, syLo, lx, wsX, waX, posX, u, v); break;
                case 6: plainFromRows<6, true>(J, sHV, sE, R, k, syLo, lx, wsX, waX, posX, u, v); break;
                default: plainFromRows<8, true>(J, sHV, sE, R, k, syLo, lx, wsX, waX, posX, u, v); break;
                }
            } else {
                switch (sup) {
                case 4: plainFromRows<4, false>(J, sHV, sE, R, k, syLo, lx, wsX, waX, posX, u, v); break;
                case 6: plainFromRows<6, false>(J, sHV, sE, R, k, syLo, lx, wsX, waX, posX, u, v); break;
                default: plainFromRows<8, false>(J, sHV, sE, R, k, syLo, lx, wsX, waX, posX, u, v); break;
                }
            }
        } else if (table && staged) {
            plainFromStaged<0>(J, sHV, sE, syLo, lx, ox, oy, u, v);
        } else {
            plainPixel(J, ox, oy, u, v);
        }
        if (floatSelector || (J.finalInTransfer && act)) {
            const size_t o = (size_t)oy * J.W + ox;
            J.oU[o] = u;                    // base for the selector blend / detail transfer
            J.oV[o] = v;
            continue;
        }
        if (J.finalInTransfer) {
            storeChroma(J, 1, ox, oy, u);
            storeChroma(J, 2, ox, oy, v);
            continue;
        }
        emit(J, ox, oy, u, v);
    }
}

__global__ void __launch_bounds__(256, 4)
k_plain(LGCR_STAGE_ARGS) {
    plainStage<false>(jobs, tileStart, njobs);
}

// the instance for launches with jinc selector frames (which often list
// every output pixel): returns at once for frames the guided pass covers
__global__ void __launch_bounds__(256, 4)
k_plain_all(LGCR_STAGE_ARGS) {
    plainStage<true>(jobs, tileStart, njobs);
}

// ---------------------------------------------------------------------------
// guided reconstruction
// ---------------------------------------------------------------------------
struct TapCtx {
    const float *lc;
    const double2 *uv;
    int cw, ch;
    float L0, nx, ny, scx, scy, rwF, rhF, invSigma2, guideFade, rescue, invG2, invG2Par;
};

struct Acc { double u, v, wsum, sumAbs; };

// One tap of pass 2 (recon.cpp:606-623). dxnx = dx*nx and dxny = (-dx)*ny
// are the per-column products of the reference's dp and dt, hoisted out of
// the row loop (same operands, same rounding). CHECKED = false when the
// caller has shown both denominators stay below 2^64 (see guidedPixel).
template <bool CHECKED>
__device__ __forceinline__ void tapCore(const TapCtx &c, float l, double2 p, float dxnx, float dxny,
                                        float dy_ny, float dy_nx, float wx, Acc &a) {
    const float dL = l - c.L0;
    const float dp = dxnx + dy_ny;
    const float dt = dxny + dy_nx;
    const float xs = 1.0f + dL * dL * c.invSigma2;
    const float simRaw = CHECKED ? rcpAtLeastOne(xs) : rcpInRange(xs);
    const float sim = 1.0f - c.guideFade * (1.0f - simRaw);
    const float xb = 1.0f + dp * dp * c.invG2 + dt * dt * c.invG2Par;
    const float bump = CHECKED ? rcpAtLeastOne(xb) : rcpInRange(xb);
    const float w = sim * (wx + c.rescue * bump);
    const double wd = (double)w;
    a.u = fma(wd, p.x, a.u);
    a.v = fma(wd, p.y, a.v);
    a.wsum += wd;
    a.sumAbs += fabs(wd);
}

__device__ __forceinline__ void tap(const TapCtx &c, size_t o, float dxf, float dy_ny, float dy_nx,
                                    float wx, Acc &a) {
    const float dx = dxf * c.rwF;
    tapCore<true>(c, ldf(c.lc + o), __ldg(c.uv + o), dx * c.nx, -dx * c.ny, dy_ny, dy_nx, wx, a);
}

// rcpInRange on both lanes: hardware approximation per lane, then the same
// fused Newton-Raphson refinement e = 1 - x*y, y' = y + y*e on the pair.
__device__ __forceinline__ f32x2 rcp2(f32x2 x, f32x2 one) {
    float x0, x1, y0, y1;
    up2(x, x0, x1);
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(x0));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y1) : "f"(x1));
    const f32x2 y = pk2(y0, y1);
    const f32x2 e = fma2(x ^ 0x8000000080000000ull, y, one);     // -x: sign bits flipped
    return fma2(y, e, y);
}

__device__ __forceinline__ void accumulate(Acc &a, float w, double2 p) {
    const double wd = (double)w;
    a.u = fma(wd, p.x, a.u);
    a.v = fma(wd, p.y, a.v);
    a.wsum += wd;
    a.sumAbs += fabs(wd);
}

// Separable base weights, all taps in range, support SUP (even; fully
// unrolled). The per-column products dx*nx and (-dx)*ny stay in registers;
// columns are processed in pairs with tapCore's arithmetic on packed pairs
// (range checks of the reciprocals hoisted by the caller), and each active
// tap is accumulated in FP64 in tap order.
// lc0/uv0 point at the window's tap (0, 0); rows are `stride` samples apart.
// SH: the window was staged in shared memory by the warp (plain loads);
// otherwise it is read from the planes in global memory.
// RADIAL: the base weight of tap (i, j) is the radial table's entry rad[j *
// SUP + i] (the jinc phase table of the output pixel) instead of wx(i) * wy(j).
template <int SUP, bool SH, bool RADIAL = false>
__device__ __forceinline__ void tapsSeparable(const TapCtx &c, int tx0, int ty0, const float *wxp,
                                              const float *wyp, uint32_t mx, uint32_t my,
                                              const float *lc0, const double2 *uv0, int stride,
                                              Acc &a, const float *rad = nullptr) {
    constexpr int NP = SUP / 2;
    f32x2 dxnx[NP], dxny[NP], wxv[NP];
    if (RADIAL) {
#pragma unroll
        for (int q = 0; q < NP; ++q)
            wxv[q] = 0ull;
    } else if (SUP % 4 == 0) {
        // the column's weights as 16-byte loads (rows of SUP floats in a
        // 256-byte aligned table)
#pragma unroll
        for (int q = 0; q < NP; q += 2) {
            const float4 w4 = __ldg(reinterpret_cast<const float4 *>(wxp) + q / 2);
            wxv[q] = pk2(w4.x, w4.y);
            wxv[q + 1] = pk2(w4.z, w4.w);
        }
    } else {
#pragma unroll
        for (int q = 0; q < NP; ++q)
            wxv[q] = pk2(__ldg(wxp + 2 * q), __ldg(wxp + 2 * q + 1));
    }
#pragma unroll
    for (int q = 0; q < NP; ++q) {
        const float dx0 = ((float)(tx0 + 2 * q) - c.scx) * c.rwF;
        const float dx1 = ((float)(tx0 + 2 * q + 1) - c.scx) * c.rwF;
        dxnx[q] = pk2(dx0 * c.nx, dx1 * c.nx);
        dxny[q] = pk2(-dx0 * c.ny, -dx1 * c.ny);
    }
    const f32x2 one = pk2(1.0f, 1.0f);
    const f32x2 L0 = pk2(c.L0, c.L0), invS = pk2(c.invSigma2, c.invSigma2);
    const f32x2 fade = pk2(c.guideFade, c.guideFade), resc = pk2(c.rescue, c.rescue);
    const f32x2 g2 = pk2(c.invG2, c.invG2), g2p = pk2(c.invG2Par, c.invG2Par);
#pragma unroll
    for (int j = 0; j < SUP; ++j) {
        if (!((my >> j) & 1u))
            continue;
        const float *lrow = lc0 + (size_t)j * stride;
        const double2 *uvrow = uv0 + (size_t)j * stride;
        const float wy = RADIAL ? 0.0f : __ldg(wyp + j);
        const float dy = ((float)(ty0 + j) - c.scy) * c.rhF;
        const f32x2 wyy = pk2(wy, wy);
        const float2 *radRow = RADIAL ? reinterpret_cast<const float2 *>(rad + j * SUP) : nullptr;
        const f32x2 dyny = pk2(dy * c.ny, dy * c.ny), dynx = pk2(dy * c.nx, dy * c.nx);
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            const int i = 2 * q;
            const double2 p0 = SH ? uvrow[i] : __ldg(uvrow + i);
            const double2 p1 = SH ? uvrow[i + 1] : __ldg(uvrow + i + 1);
            const float l0 = SH ? lrow[i] : ldf(lrow + i), l1 = SH ? lrow[i + 1] : ldf(lrow + i + 1);
            const f32x2 dL = sub2(pk2(l0, l1), L0);
            const f32x2 simRaw = rcp2(add2(one, mul2(mul2(dL, dL), invS)), one);
            const f32x2 sim = sub2(one, mul2(fade, sub2(one, simRaw)));
            const f32x2 dp = add2(dxnx[q], dyny);
            const f32x2 dt = add2(dxny[q], dynx);
            const f32x2 bump = rcp2(add2(add2(one, mul2(mul2(dp, dp), g2)), mul2(mul2(dt, dt), g2p)), one);
            f32x2 base;
            if (RADIAL) {
                const float2 r2 = __ldg(radRow + q);
                base = pk2(r2.x, r2.y);
            } else {
                base = mul2(wxv[q], wyy);
            }
            const f32x2 w = mul2(sim, add2(base, mul2(resc, bump)));
            float w0, w1;
            up2(w, w0, w1);
            if ((mx >> i) & 1u)
                accumulate(a, w0, p0);
            if ((mx >> (i + 1)) & 1u)
                accumulate(a, w1, p1);
        }
    }
}

// Any support, clamped taps; separable or radial base weights.
__device__ __forceinline__ void tapsGeneric(const FrameJob &J, const TapCtx &c, int ox, int oy,
                                            int tx0, int ty0, Acc &a) {
    const AxisView &ax = J.ax, &ay = J.ay;
    const float *wxp = ax.w + (size_t)ox * ax.sup;
    const uint8_t *amx = ax.am + (size_t)ox * ax.sup;
    const float *wyp = ay.w + (size_t)oy * ay.sup;
    const uint8_t *amy = ay.am + (size_t)oy * ay.sup;
    const float *base = J.radial ? radialWeightsAt(J.rad, ox, oy) : nullptr;
    for (int j = 0; j < ay.sup; ++j) {
        if (__ldg(amy + j) == 0)
            continue;
        const size_t rowOff = (size_t)iclamp(ty0 + j, 0, c.ch - 1) * c.cw;
        const float wy = __ldg(wyp + j);
        const float dyf = (float)(ty0 + j) - c.scy;
        const float dy = dyf * c.rhF;
        const float dyc = dyf * J.invWyC;
        const float dy_ny = dy * c.ny, dy_nx = dy * c.nx;
        for (int i = 0; i < ax.sup; ++i) {
            if (__ldg(amx + i) == 0)
                continue;
            const size_t o = rowOff + iclamp(tx0 + i, 0, c.cw - 1);
            const float dxf = (float)(tx0 + i) - c.scx;
            float wx;
            if (base) {
                wx = ldf(base + (size_t)j * ax.sup + i);
            } else if (J.radial) {
                const float dxc = dxf * J.invWxC;
                wx = lutLookupDev(J.lut, J.lutN, sqrtf(dxc * dxc + dyc * dyc) * J.lutScale);
            } else {
                wx = __ldg(wxp + i) * wy;
            }
            tap(c, o, dxf, dy_ny, dy_nx, wx, a);
        }
    }
}

// Window extrema of U, V and lc over the active taps from the table rows:
// ext = {minU, maxU, minV, maxV, minL, maxL}.
template <int SUP>
__device__ __forceinline__ void windowExtrema(const FrameJob &J, int ox, int ty0, const uint8_t *amy,
                                              float *ext) {
    const int n = SUP > 0 ? SUP : J.ay.sup;
    float mnU = 1e30f, mxU = -1e30f, mnV = 1e30f, mxV = -1e30f, mnL = 1e30f, mxL = -1e30f;
#pragma unroll
    for (int j = 0; j < n; ++j) {
        if (__ldg(amy + j) == 0)
            continue;
        const int sy = J.noClampY ? ty0 + j : iclamp(ty0 + j, 0, J.ch - 1);
        const float4 *h = reinterpret_cast<const float4 *>(J.hTab + ((size_t)sy * J.W + ox) * 8);
        const float4 a = __ldg(h), b = __ldg(h + 1);
        mnU = runMin(mnU, a.z); mxU = runMax(mxU, a.w);
        mnV = runMin(mnV, b.x); mxV = runMax(mxV, b.y);
        mnL = runMin(mnL, b.z); mxL = runMax(mxL, b.w);
    }
    ext[0] = mnU; ext[1] = mxU; ext[2] = mnV; ext[3] = mxV; ext[4] = mnL; ext[5] = mxL;
}

// Pass 1 of the guided pixel over a window whose taps are all in range:
// h = {max |lc - L0|, min U, max U, min V, max V} over the active taps, in
// the generic loop's order (rows, then columns) with bit masks and no
// clamping.
template <int SUP>
__device__ __forceinline__ void windowHullInRange(const FrameJob &J, int tx0, int ty0,
                                                  const uint8_t *amx, const uint8_t *amy, float L0,
                                                  float *h) {
    const uint32_t mx = maskBits(amx, SUP), my = maskBits(amy, SUP);
    float maxAbsDL = 0.0f, mnU = 1e30f, mxU = -1e30f, mnV = 1e30f, mxV = -1e30f;
#pragma unroll
    for (int j = 0; j < SUP; ++j) {
        if (!((my >> j) & 1u))
            continue;
        const size_t row = (size_t)(ty0 + j) * J.cw + tx0;
#pragma unroll
        for (int i = 0; i < SUP; ++i) {
            if (!((mx >> i) & 1u))
                continue;
            const float l = ldf(J.lc + row + i), u = ldf(J.U + row + i), v = ldf(J.V + row + i);
            maxAbsDL = smax(maxAbsDL, fabsf(l - L0));
            mnU = smin(mnU, u); mxU = smax(mxU, u);
            mnV = smin(mnV, v); mxV = smax(mxV, v);
        }
    }
    h[0] = maxAbsDL; h[1] = mnU; h[2] = mxU; h[3] = mnV; h[4] = mxV;
}

// Pass 1 fused with the radial plain base of the same window (jinc frames
// whose selector needs the plain sample): the active taps are the plain
// pass's too (same axis activity and window start), so one traversal gives
// the guided hull and luma range and the plain sums of plainRadialTable
// (phase-table weights, FP64 in the same tap order). The hull comes from
// the FP64 copies of the samples (the same values as the float planes).
struct RadialPlainSums {
    double u, v, wsum, sumAbs;
};

template <int SUP>
__device__ __forceinline__ void windowHullPlainRadial(const FrameJob &J, int tx0, int ty0,
                                                      const uint8_t *amx, const uint8_t *amy, float L0,
                                                      const float *base, float *h, RadialPlainSums &ps) {
    const uint32_t mx = maskBits(amx, SUP), my = maskBits(amy, SUP);
    const double2 *uvd = reinterpret_cast<const double2 *>(J.uvd);
    float maxAbsDL = 0.0f;
    double mnU = 1e30, mxU = -1e30, mnV = 1e30, mxV = -1e30;
    double au = 0.0, av = 0.0, ws = 0.0, wa = 0.0;
#pragma unroll
    for (int j = 0; j < SUP; ++j) {
        if (!((my >> j) & 1u))
            continue;
        const size_t row = (size_t)(ty0 + j) * J.cw + tx0;
        const float2 *wrow = reinterpret_cast<const float2 *>(base + j * SUP);
#pragma unroll
        for (int q = 0; q < SUP / 2; ++q) {
            const float2 w2 = __ldg(wrow + q);
            const float wk[2] = { w2.x, w2.y };
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int i = 2 * q + k;
                if (!((mx >> i) & 1u))
                    continue;
                const float l = ldf(J.lc + row + i);
                const double2 p = __ldg(uvd + row + i);
                maxAbsDL = smax(maxAbsDL, fabsf(l - L0));
                mnU = smin(mnU, p.x); mxU = smax(mxU, p.x);
                mnV = smin(mnV, p.y); mxV = smax(mxV, p.y);
                const double wd = (double)wk[k];
                au = fma(wd, p.x, au);
                av = fma(wd, p.y, av);
                ws += wd;
                wa += fabs(wd);
            }
        }
    }
    h[0] = maxAbsDL; h[1] = (float)mnU; h[2] = (float)mxU; h[3] = (float)mnV; h[4] = (float)mxV;
    ps.u = au; ps.v = av; ps.wsum = ws; ps.sumAbs = wa;
}

struct Guided {
    double u, v;
    float L0, ssRamp, guideFade, nx, ny;
    bool hasDir;
    bool havePlain;                     // plainU/V hold the plain base
    float plainU, plainV;
};

// A warp's guided-tap window staged in shared memory: kStageRows x
// kStageCols chroma samples (lc and the FP64 (u, v) pair) starting at chroma
// (tx0, ty0), the same rows for every pixel of the warp.
constexpr int kStageRows = 8, kStageCols = 40;
struct StagedWindow {
    const float *lc;
    const double2 *uv;
    int tx0, ty0;
};

// RFUSE: the kernel instance for batches with jinc selector frames (their
// pass 1 also forms the plain base); the other instance has no such code, so
// the separable frames' tap loops keep their schedule. RONLY: launches whose
// frames are all such jinc frames; the separable, extrema-table and
// temporal paths are compiled out, which leaves the 3-blocks budget far
// fewer spills.
template <bool RFUSE, bool RONLY = false>
__device__ __forceinline__ Guided guidedPixel(const FrameJob &J, int ox, int oy,
                                              const StagedWindow *win) {
    const AxisView &ax = J.ax, &ay = J.ay;
    const int sw = J.sw, sh = J.sh, cw = J.cw, ch = J.ch;
    Guided g;
    // window extrema folded by k_plain (issued first: nothing else waits on them)
    float4 wHull = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float2 wLum = make_float2(0.0f, 0.0f);
    if (J.wHull) {
        const size_t o = (size_t)oy * J.W + ox;
        wHull = __ldg(J.wHull + o);
        wLum = __ldg(J.wLum + o);
    }
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

    // pass 1: window luma range and chroma hull over the active taps. The
    // luma range max|lc - L0| equals max(|max lc - L0|, |min lc - L0|)
    // exactly (float subtraction is monotonic), so the table's extrema serve.
    const int tx0 = __ldg(ax.start + ox), ty0 = __ldg(ay.start + oy);
    const float *wxp = ax.w + (size_t)ox * ax.sup;
    const uint8_t *amx = ax.am + (size_t)ox * ax.sup;
    const float *wyp = ay.w + (size_t)oy * ay.sup;
    const uint8_t *amy = ay.am + (size_t)oy * ay.sup;
    float maxAbsDL = 0.0f;
    float hMinU = 1e30f, hMaxU = -1e30f, hMinV = 1e30f, hMaxV = -1e30f;
    g.havePlain = false;
    g.plainU = g.plainV = 0.0f;
    // jinc selector frames: the plain base of the listed pixels comes from
    // this pass (the plain stage skips them)
    const bool fusePlain = RFUSE && radialPlainFused(J);
    if (fusePlain) {
        float h[5];
        RadialPlainSums ps;
        const float *rbase = radialWeightsAt(J.rad, ox, oy);
        switch (ax.sup) {
        case 4: windowHullPlainRadial<4>(J, tx0, ty0, amx, amy, L0, rbase, h, ps); break;
        case 6: windowHullPlainRadial<6>(J, tx0, ty0, amx, amy, L0, rbase, h, ps); break;
        default: windowHullPlainRadial<8>(J, tx0, ty0, amx, amy, L0, rbase, h, ps); break;
        }
        maxAbsDL = h[0]; hMinU = h[1]; hMaxU = h[2]; hMinV = h[3]; hMaxV = h[4];
        // the plain base's finish (plainRadialTable in plain.cuh)
        double v0, v1;
        if (ps.wsum > 1e-6 && ps.wsum >= 0.05 * ps.sumAbs) {
            v0 = ps.u / ps.wsum;
            v1 = ps.v / ps.wsum;
        } else {
            v0 = bilinearAt(J.U, cw, ch, __ldg(ax.pos + ox), __ldg(ay.pos + oy));
            v1 = bilinearAt(J.V, cw, ch, __ldg(ax.pos + ox), __ldg(ay.pos + oy));
        }
        if (J.clampHull) {
            v0 = sclamp(v0, (double)(hMinU - J.margin), (double)(hMaxU + J.margin));
            v1 = sclamp(v1, (double)(hMinV - J.margin), (double)(hMaxV + J.margin));
        }
        g.havePlain = true;
        g.plainU = (float)v0;
        g.plainV = (float)v1;
    } else if (!RONLY && J.wHull) {
        hMinU = wHull.x; hMaxU = wHull.y; hMinV = wHull.z; hMaxV = wHull.w;
        maxAbsDL = smax(maxAbsDL, fabsf(wLum.y - L0));
        maxAbsDL = smax(maxAbsDL, fabsf(wLum.x - L0));
    } else if (!RONLY && !J.radial && J.hTab) {
        float ext[6];
        switch (ay.sup) {
        case 4: windowExtrema<4>(J, ox, ty0, amy, ext); break;
        case 6: windowExtrema<6>(J, ox, ty0, amy, ext); break;
        case 8: windowExtrema<8>(J, ox, ty0, amy, ext); break;
        default: windowExtrema<0>(J, ox, ty0, amy, ext); break;
        }
        hMinU = ext[0]; hMaxU = ext[1]; hMinV = ext[2]; hMaxV = ext[3];
        maxAbsDL = smax(maxAbsDL, fabsf(ext[5] - L0));
        maxAbsDL = smax(maxAbsDL, fabsf(ext[4] - L0));
    } else if (J.noClampX && J.noClampY && ax.sup == ay.sup &&
               (ax.sup == 4 || ax.sup == 6 || ax.sup == 8)) {
        float h[5];
        switch (ax.sup) {
        case 4: windowHullInRange<4>(J, tx0, ty0, amx, amy, L0, h); break;
        case 6: windowHullInRange<6>(J, tx0, ty0, amx, amy, L0, h); break;
        default: windowHullInRange<8>(J, tx0, ty0, amx, amy, L0, h); break;
        }
        maxAbsDL = h[0]; hMinU = h[1]; hMaxU = h[2]; hMinV = h[3]; hMaxV = h[4];
    } else {
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
                // per-axis max |w| and sum of w^2 over the active taps (host tables
                // of the same float sums)
                const float mxX = __ldg(ax.kmx + ox), ssX = __ldg(ax.kss + ox);
                const float mxY = __ldg(ay.kmx + oy), ssY = __ldg(ay.kss + oy);
                kappa = (mxX * mxX * mxY * mxY) / (ssX * ssY + 1e-12f);
            } else if (J.rad.valid && J.rad.kappa) {
                // the phase table's kappa: the same float sums over the
                // phase's active taps, evaluated once per phase on the host
                const size_t phase = (size_t)__ldg(J.rad.yPhase + oy) * J.rad.phasesX +
                                     __ldg(J.rad.xPhase + ox);
                kappa = ldf(J.rad.kappa + phase);
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

    // pass 2: taps with w = sim * (wbase + rescue * bump)
    TapCtx c;
    c.lc = J.lc;
    c.uv = reinterpret_cast<const double2 *>(J.uvd);
    c.cw = cw; c.ch = ch;
    c.L0 = L0; c.nx = nx; c.ny = ny; c.scx = scx; c.scy = scy;
    c.rwF = J.rwF; c.rhF = J.rhF;
    c.invSigma2 = invSigma2; c.guideFade = guideFade; c.rescue = rescue;
    c.invG2 = J.invGsigma2;
    c.invG2Par = J.invGsigma2 / (aniso * aniso);
    Acc a{0.0, 0.0, 0.0, 0.0};
    // The unrolled loops skip the reciprocal's range check: every tap's
    // similarity denominator 1 + dL^2/sigma^2 is at most the same expression
    // at the window's luma range maxAbsDL (each rounding step is monotonic),
    // and the frame's bump denominators are bounded on the host.
    const bool rcpSafe = J.bumpRcpSafe && (1.0f + maxAbsDL * maxAbsDL * invSigma2) < kRcpFastLimit;
    const bool fast = !RONLY && !J.radial && J.noClampX && J.noClampY && ax.sup == ay.sup && rcpSafe;
    // jinc with a phase table: the same unrolled loop with table weights
    const bool fastRadial = J.radial && J.rad.valid && J.rad.supX == ax.sup && J.rad.supY == ay.sup &&
                            J.noClampX && J.noClampY && ax.sup == ay.sup && rcpSafe &&
                            (ax.sup == 4 || ax.sup == 6 || ax.sup == 8);
    if (fast && win) {
        // the warp staged rows ty0 .. ty0 + sup - 1 around every pixel's columns
        const float *l0 = win->lc + (tx0 - win->tx0);
        const double2 *u0 = win->uv + (tx0 - win->tx0);
        if (ax.sup == 8)
            tapsSeparable<8, true>(c, tx0, ty0, wxp, wyp,
                                   ax.amBits ? __ldg(ax.amBits + ox) : maskBits(amx, 8),
                                   ay.amBits ? __ldg(ay.amBits + oy) : maskBits(amy, 8),
                                   l0, u0, kStageCols, a);
        else if (ax.sup == 6)
            tapsSeparable<6, true>(c, tx0, ty0, wxp, wyp, maskBits(amx, 6), maskBits(amy, 6),
                                   l0, u0, kStageCols, a);
        else
            tapsSeparable<4, true>(c, tx0, ty0, wxp, wyp, maskBits(amx, 4), maskBits(amy, 4),
                                   l0, u0, kStageCols, a);
    } else if (fast && ax.sup <= 8 && !(ax.sup & 1) && ax.sup >= 4) {
        const float *l0 = c.lc + (size_t)ty0 * c.cw + tx0;
        const double2 *u0 = c.uv + (size_t)ty0 * c.cw + tx0;
        if (ax.sup == 8)
            tapsSeparable<8, false>(c, tx0, ty0, wxp, wyp,
                                    ax.amBits ? __ldg(ax.amBits + ox) : maskBits(amx, 8),
                                    ay.amBits ? __ldg(ay.amBits + oy) : maskBits(amy, 8),
                                    l0, u0, c.cw, a);
        else if (ax.sup == 6)
            tapsSeparable<6, false>(c, tx0, ty0, wxp, wyp, maskBits(amx, 6), maskBits(amy, 6),
                                    l0, u0, c.cw, a);
        else
            tapsSeparable<4, false>(c, tx0, ty0, wxp, wyp, maskBits(amx, 4), maskBits(amy, 4),
                                    l0, u0, c.cw, a);
    } else if (fastRadial && win) {
        // the warp staged rows ty0 .. ty0 + sup - 1 around every pixel's columns
        const float *l0 = win->lc + (tx0 - win->tx0);
        const double2 *u0 = win->uv + (tx0 - win->tx0);
        const float *rad = radialWeightsAt(J.rad, ox, oy);
        if (ax.sup == 6)
            tapsSeparable<6, true, true>(c, tx0, ty0, nullptr, nullptr, maskBits(amx, 6),
                                         maskBits(amy, 6), l0, u0, kStageCols, a, rad);
        else if (ax.sup == 8)
            tapsSeparable<8, true, true>(c, tx0, ty0, nullptr, nullptr, maskBits(amx, 8),
                                         maskBits(amy, 8), l0, u0, kStageCols, a, rad);
        else
            tapsSeparable<4, true, true>(c, tx0, ty0, nullptr, nullptr, maskBits(amx, 4),
                                         maskBits(amy, 4), l0, u0, kStageCols, a, rad);
    } else if (fastRadial) {
        const float *l0 = c.lc + (size_t)ty0 * c.cw + tx0;
        const double2 *u0 = c.uv + (size_t)ty0 * c.cw + tx0;
        const float *rad = radialWeightsAt(J.rad, ox, oy);
        if (ax.sup == 6)
            tapsSeparable<6, false, true>(c, tx0, ty0, nullptr, nullptr, maskBits(amx, 6),
                                          maskBits(amy, 6), l0, u0, c.cw, a, rad);
        else if (ax.sup == 8)
            tapsSeparable<8, false, true>(c, tx0, ty0, nullptr, nullptr, maskBits(amx, 8),
                                          maskBits(amy, 8), l0, u0, c.cw, a, rad);
        else
            tapsSeparable<4, false, true>(c, tx0, ty0, nullptr, nullptr, maskBits(amx, 4),
                                          maskBits(amy, 4), l0, u0, c.cw, a, rad);
    } else {
        tapsGeneric(J, c, ox, oy, tx0, ty0, a);
    }
    if (!RONLY && J.tnbCount > 0) {
        // TRecon: the neighbours' motion-compensated samples follow the
        // spatial taps in the same accumulators and extend the hull
        TemporalAcc t{a.u, a.v, a.wsum, a.sumAbs, hMinU, hMaxU, hMinV, hMaxV};
        t = temporalTaps(J, ox, oy, L0, scx, scy, sigLoc, guideFade, ssRamp, t);
        a.u = t.u; a.v = t.v; a.wsum = t.wsum; a.sumAbs = t.sumAbs;
        hMinU = t.mnU; hMaxU = t.mxU; hMinV = t.mnV; hMaxV = t.mxV;
    }

    double valueU, valueV;
    if (a.wsum > 1e-6 && a.wsum >= 0.05 * a.sumAbs) {
        valueU = a.u / a.wsum;
        valueV = a.v / a.wsum;
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

// One listed pixel: algo 2 output, or the algo 4 selector (recon.cpp:762-811).
template <bool RFUSE, bool RONLY>
__device__ __forceinline__ void guidedWork(const FrameJob &J, int ox, int oy,
                                           const StagedWindow *win) {
    const Guided g = guidedPixel<RFUSE, RONLY>(J, ox, oy, win);
    if (J.algo == 2) {
        emit(J, ox, oy, (float)g.u, (float)g.v);
        return;
    }
    const float diag = g.hasDir ? smin(1.0f, 2.0f * fabsf(g.nx * g.ny)) : 0.0f;
    const float hedgy = (1.0f - g.ssRamp) * g.guideFade;
    const float sel = J.strength4;
    const float w2 = hedgy * (1.0f - diag) * sel;
    const float w3 = hedgy * diag * sel;
    const size_t o = (size_t)oy * J.W + ox;
    if (J.outKind != kF32) {
        // integer output: single-expression fused selector on the plain base
        float baseU, baseV;
        if (RFUSE && g.havePlain) {
            baseU = g.plainU;
            baseV = g.plainV;
        } else {
            plainPixel(J, ox, oy, baseU, baseV);
        }
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
    float baseU, baseV;
    if (RFUSE && g.havePlain) {
        // the plain base of this listed pixel, for the blend stage too
        baseU = g.plainU;
        baseV = g.plainV;
        J.oU[o] = baseU;
        J.oV[o] = baseV;
    } else {
        baseU = J.oU[o];
        baseV = J.oV[o];
    }
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

// Persistent grid over the work lists of all frames in the launch. Each
// block builds the prefix of the frames' list lengths in shared memory and
// strides over the concatenated work, a warp taking 32 consecutive entries.
//
// STAGED: when a warp's 32 pixels are one frame's separable, unclamped fast
// taps and share their chroma rows (one output row, as both list orders
// mostly give: a warp's 32 entries are one 32-pixel word of one row wherever
// the frame is dense) with at most kStageCols columns between the first and
// last window, the warp first copies that window of lc and (u, v) into its
// shared-memory slice with cp.async (global -> shared, no register round
// trip); the taps then read shared memory. The values and the arithmetic
// are the same either way.
constexpr int kGuidedMaxFrames = 1024;

// cp.async copies of 4 and 16 bytes (both addresses aligned to the size)
__device__ __forceinline__ void cpAsync4(void *smem, const void *gmem) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" :: "r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpAsync16(void *smem, const void *gmem) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" :: "r"(dst), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cpAsyncWaitAll() {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

static_assert(kGuidedStageBytes == size_t(8) * kStageRows * kStageCols * (4 + 16),
              "staged guided windows: 8 warps x kStageRows x kStageCols x (lc + (u, v))");

template <int MIN_BLOCKS, bool STAGED, bool RFUSE, bool RONLY = false>
__device__ __forceinline__ void guidedGrid(const FrameJob *__restrict__ jobs, int njobs) {
    __shared__ unsigned long long pre[kGuidedMaxFrames + 1];
    extern __shared__ __align__(16) unsigned char guidedStage[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double2 *sUv = reinterpret_cast<double2 *>(guidedStage) + warp * (kStageRows * kStageCols);
    float *sLc = reinterpret_cast<float *>(guidedStage + size_t(8) * kStageRows * kStageCols * 16) +
                 warp * (kStageRows * kStageCols);
    for (int chunk = 0; chunk < njobs; chunk += kGuidedMaxFrames) {
        const int n = min(kGuidedMaxFrames, njobs - chunk);
        if (threadIdx.x == 0) {
            unsigned long long acc = 0;
            for (int i = 0; i < n; ++i) {
                pre[i] = acc;
                const FrameJob &J = jobs[chunk + i];
                if (J.listed)
                    acc += J.counters[kCntActiveOutput];
            }
            pre[n] = acc;
        }
        __syncthreads();
        const unsigned long long total = pre[n];
        const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
        for (unsigned long long wb = (unsigned long long)blockIdx.x * blockDim.x + warp * 32;
             wb < total; wb += stride) {
            const unsigned long long w = wb + lane;
            const bool valid = w < total;
            int lo = 0;
            if (valid) {
                int hi = n - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (pre[mid] <= w) lo = mid; else hi = mid - 1;
                }
            }
            const FrameJob &J = jobs[chunk + lo];
            const uint32_t pix = valid ? J.actList[w - pre[lo]] : 0u;
            const int ox = (int)(pix & 0xffffu), oy = (int)(pix >> 16);
            StagedWindow sw;
            const StagedWindow *win = nullptr;
            if (STAGED) {
                const bool all = __all_sync(0xffffffffu, valid);
                const int loMin = __reduce_min_sync(0xffffffffu, lo);
                const int loMax = __reduce_max_sync(0xffffffffu, lo);
                const int sup = J.ax.sup;
                // separable frames, and jinc frames with a phase table (the
                // radial tap loop reads the same staged window)
                const bool radialOk = !J.radial || (J.rad.valid && J.rad.supX == sup && J.rad.supY == sup);
                bool ok = all && loMin == loMax && radialOk && J.noClampX && J.noClampY &&
                          sup == J.ay.sup && sup <= kStageRows && sup >= 4 && !(sup & 1);
                int tx0 = 0, ty0 = 0, txMin = 0, txMax = 0, tyMin = 0, tyMax = 0;
                if (ok) {                                   // warp-uniform
                    tx0 = __ldg(J.ax.start + ox);
                    ty0 = __ldg(J.ay.start + oy);
                    txMin = __reduce_min_sync(0xffffffffu, tx0);
                    txMax = __reduce_max_sync(0xffffffffu, tx0);
                    tyMin = __reduce_min_sync(0xffffffffu, ty0);
                    tyMax = __reduce_max_sync(0xffffffffu, ty0);
                    ok = tyMin == tyMax && txMax + sup - txMin <= kStageCols;
                }
                if (ok) {
                    // every index in range: starts lie in [0, n - sup] (noClamp)
                    const int cols = txMax + sup - txMin;
                    const double2 *uvd = reinterpret_cast<const double2 *>(J.uvd);
                    // asynchronous global -> shared copies (no register round
                    // trip); the warp waits for its own copies, then syncs
                    for (int k = lane; k < sup * cols; k += 32) {
                        const int r = k / cols, cc = k - r * cols;
                        const size_t g = (size_t)(tyMin + r) * J.cw + txMin + cc;
                        cpAsync4(sLc + r * kStageCols + cc, J.lc + g);
                        cpAsync16(sUv + r * kStageCols + cc, uvd + g);
                    }
                    cpAsyncWaitAll();
                    __syncwarp();
                    sw.lc = sLc;
                    sw.uv = sUv;
                    sw.tx0 = txMin;
                    sw.ty0 = tyMin;
                    win = &sw;
                }
            }
            if (valid)
                guidedWork<RFUSE, RONLY>(J, ox, oy, win);
            if (STAGED)
                __syncwarp();                       // the slice is rewritten next round
        }
        __syncthreads();
    }
}

// Register budgets of the same persistent kernel: 2 resident blocks per SM
// (no spills) or 3 (fewer registers, a few spills), and 2 blocks with the
// warps' tap windows (separable or jinc) staged in shared memory; the
// autotuner picks.
__global__ void __launch_bounds__(256, 2)
k_guided(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    guidedGrid<2, false, false>(jobs, njobs);
}

__global__ void __launch_bounds__(256, 3)
k_guided3(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    guidedGrid<3, false, false>(jobs, njobs);
}

__global__ void __launch_bounds__(256, 2)
k_guided_staged(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    guidedGrid<2, true, false>(jobs, njobs);
}

// the same three for batches with jinc selector frames
__global__ void __launch_bounds__(256, 2)
k_guided_r(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    guidedGrid<2, false, true>(jobs, njobs);
}

__global__ void __launch_bounds__(256, 3)
k_guided3_r(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    guidedGrid<3, false, true>(jobs, njobs);
}

__global__ void __launch_bounds__(256, 2)
k_guided_staged_r(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    guidedGrid<2, true, true>(jobs, njobs);
}

// and for launches of jinc selector frames only
__global__ void __launch_bounds__(256, 2)
k_guided_o(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    guidedGrid<2, false, true, true>(jobs, njobs);
}

__global__ void __launch_bounds__(256, 3)
k_guided3_o(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    guidedGrid<3, false, true, true>(jobs, njobs);
}

__global__ void __launch_bounds__(256, 2)
k_guided_staged_o(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    (void)tileStart;
    guidedGrid<2, true, true, true>(jobs, njobs);
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

// 2D jinc luma resize (resampleRadial, src/kernels.cpp:276-334). A 32x32
// tile of output pixels (256 threads, four rows each) stages the clamped
// input rows and columns its windows cover, as doubles (the accumulation's
// operand type). A tap's weight
// depends only on the pixel's column offsets (x0 + i - cx) / widen and row
// offsets (y0 + j - cy) / widen as floats, so warp 0 groups the block's
// columns (and rows) whose offset vectors are identical, the block evaluates
// the weights once per (column group, row group) into a shared table of
// doubles, and every pixel accumulates from shared memory: one weight load,
// one sample load and one FP64 FMA per tap. Blocks whose groups do not fit
// the table evaluate each tap per pixel. The weights, their order and the
// FP64 accumulation are the reference's.
constexpr int kRadialBx = 32, kRadialBy = 32; // output tile of one block
constexpr int kRadialTileMax = 2048;         // staged luma samples per block
constexpr int kRadialMaxSup = 16;            // offsets kept per column / row
constexpr int kRadialWeightsMax = 1152;      // shared weight table (doubles)

template <int SUP>
__device__ __forceinline__ void radialTabled(const double *__restrict__ w, const double *__restrict__ s,
                                             int fw, double &acc, double &wsum) {
#pragma unroll
    for (int j = 0; j < SUP; ++j) {
#pragma unroll
        for (int i = 0; i < SUP; ++i) {
            const double wv = w[j * SUP + i];
            acc = fma(wv, s[j * fw + i], acc);
            wsum += wv;
        }
    }
}

__global__ void __launch_bounds__(256)
k_luma_radial(const FrameJob *__restrict__ jobs, const int *__restrict__ tileStart, int njobs) {
    __shared__ double sY[kRadialTileMax];
    __shared__ double sW[kRadialWeightsMax];
    __shared__ float sDx[kRadialBx][kRadialMaxSup], sDy[kRadialBy][kRadialMaxSup];
    __shared__ int sColIdx[kRadialBx], sRowIdx[kRadialBy], sColRep[kRadialBx], sRowRep[kRadialBy];
    __shared__ int sColN, sRowN;
    const int f = findFrame(tileStart, njobs, blockIdx.x);
    const FrameJob &J = jobs[f];
    const int tile = blockIdx.x - tileStart[f];
    const int tilesX = (J.W + kRadialBx - 1) / kRadialBx;
    const int bx0 = (tile % tilesX) * kRadialBx, by0 = (tile / tilesX) * kRadialBy;
    const int ox = bx0 + threadIdx.x;
    const double sx = (double)J.sw / J.W, sy = (double)J.sh / J.H;
    const double widen = fmax(1.0, fmax(sx, sy));
    const float invW = (float)(1.0 / widen);
    const int radius = (int)ceil(J.support * widen);
    const int sup = 2 * radius;
    // the block's footprint: first tap of its first pixel to last tap of its
    // last pixel, per axis (the first tap grows with the output index)
    const int bxLast = min(bx0 + kRadialBx - 1, J.W - 1), byLast = min(by0 + kRadialBy - 1, J.H - 1);
    const int fx0 = (int)ceil((bx0 + 0.5) * sx - 0.5 - radius);
    const int fy0 = (int)ceil((by0 + 0.5) * sy - 0.5 - radius);
    const int fw = (int)ceil((bxLast + 0.5) * sx - 0.5 - radius) + sup - fx0;
    const int fh = (int)ceil((byLast + 0.5) * sy - 0.5 - radius) + sup - fy0;
    const bool tileStaged = fw * fh <= kRadialTileMax;
    const bool grouped = tileStaged && sup <= kRadialMaxSup;
    const int nt = blockDim.x * blockDim.y, t = threadIdx.y * blockDim.x + threadIdx.x;
    if (tileStaged)
        for (int k = t; k < fw * fh; k += nt)
            sY[k] = (double)ldf(J.Y + (size_t)iclamp(fy0 + k / fw, 0, J.sh - 1) * J.sw +
                                iclamp(fx0 + k % fw, 0, J.sw - 1));
    const double cx = (ox + 0.5) * sx - 0.5;
    const int x0 = (int)ceil(cx - radius);
    if (grouped && threadIdx.y == 0) {
        // warp 0: lane l holds column l's offsets and row l's; each column
        // (row) joins the group of its first identical predecessor
        const int lane = threadIdx.x;
        for (int i = 0; i < sup; ++i)
            sDx[lane][i] = (float)((x0 + i - cx) * invW);
        const double ry = (by0 + lane + 0.5) * sy - 0.5;
        const int ry0 = (int)ceil(ry - radius);
        for (int j = 0; j < sup; ++j)
            sDy[lane][j] = (float)((ry0 + j - ry) * invW);
        __syncwarp();
        int c = lane, r = lane;
        for (int q = 0; q < lane && c == lane; ++q) {
            bool same = true;
            for (int i = 0; i < sup && same; ++i)
                same = __float_as_uint(sDx[q][i]) == __float_as_uint(sDx[lane][i]);
            if (same)
                c = q;
        }
        for (int q = 0; q < lane && r == lane; ++q) {
            bool same = true;
            for (int j = 0; j < sup && same; ++j)
                same = __float_as_uint(sDy[q][j]) == __float_as_uint(sDy[lane][j]);
            if (same)
                r = q;
        }
        const unsigned below = (1u << lane) - 1u;
        const unsigned colReps = __ballot_sync(0xffffffffu, c == lane);
        const unsigned rowReps = __ballot_sync(0xffffffffu, r == lane);
        // group number = rank of the representative among the representatives
        const int myCol = __popc(colReps & below), myRow = __popc(rowReps & below);
        sColIdx[lane] = __shfl_sync(0xffffffffu, myCol, c);
        sRowIdx[lane] = __shfl_sync(0xffffffffu, myRow, r);
        if (c == lane)
            sColRep[myCol] = lane;
        if (r == lane)
            sRowRep[myRow] = lane;
        if (lane == 0) {
            sColN = __popc(colReps);
            sRowN = __popc(rowReps);
        }
    }
    __syncthreads();
    bool tabled = false;
    if (grouped) {
        const int nc = sColN, nr = sRowN, per = sup * sup;
        tabled = nc * nr * per <= kRadialWeightsMax;
        if (tabled)
            for (int k = t; k < nc * nr * per; k += nt) {
                const int pair = k / per, tap = k - pair * per;
                const int qc = sColRep[pair % nc], qr = sRowRep[pair / nc];
                const float dx = sDx[qc][tap % sup], dy = sDy[qr][tap / sup];
                sW[k] = (double)lutLookupDev(J.lut, J.lutN, sqrtf(dx * dx + dy * dy) * J.lutScale);
            }
        __syncthreads();
    }
    if (ox >= J.W)
        return;
    // each thread: the rows threadIdx.y, + 8, + 16, + 24 of its column
    for (int ly = threadIdx.y; ly < kRadialBy; ly += blockDim.y) {
        const int oy = by0 + ly;
        if (oy >= J.H)
            break;
        const double cy = (oy + 0.5) * sy - 0.5;
        const int y0 = (int)ceil(cy - radius);
        double acc = 0.0, wsum = 0.0;
        if (tabled) {
            const double *w = sW + (size_t)(sRowIdx[ly] * sColN + sColIdx[threadIdx.x]) * sup * sup;
            const double *s = sY + (y0 - fy0) * fw + (x0 - fx0);
            if (sup == 6) {
                radialTabled<6>(w, s, fw, acc, wsum);
            } else if (sup == 4) {
                radialTabled<4>(w, s, fw, acc, wsum);
            } else if (sup == 8) {
                radialTabled<8>(w, s, fw, acc, wsum);
            } else {
                for (int j = 0; j < sup; ++j)
                    for (int i = 0; i < sup; ++i) {
                        const double wv = w[j * sup + i];
                        acc = fma(wv, s[j * fw + i], acc);
                        wsum += wv;
                    }
            }
        } else {
            for (int j = 0; j < sup; ++j) {
                const float dy = (float)((y0 + j - cy) * invW);
                const int srow = (y0 + j - fy0) * fw - fx0;
                const float *row = J.Y + (size_t)iclamp(y0 + j, 0, J.sh - 1) * J.sw;
                for (int i = 0; i < sup; ++i) {
                    const float dx = (float)((x0 + i - cx) * invW);
                    const float w = lutLookupDev(J.lut, J.lutN, sqrtf(dx * dx + dy * dy) * J.lutScale);
                    const double v = tileStaged ? sY[srow + x0 + i]
                                                : (double)ldf(row + iclamp(x0 + i, 0, J.sw - 1));
                    acc = fma((double)w, v, acc);
                    wsum += (double)w;
                }
            }
        }
        storeLuma(J, ox, oy, (float)(wsum > 1e-6 ? acc / wsum : 0.0));
    }
}


} // namespace lgcr_b200
