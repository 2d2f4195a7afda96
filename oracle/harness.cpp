// oracle/harness.cpp — TEST INFRASTRUCTURE ONLY (the oracle).
//
// Restates the per-frame orchestration of the reference's Recon, Sharpen and
// TRecon filters over raw planar host buffers, so that the reference's own
// compute functions (compiled unmodified from src/{maps,kernels,recon,algos,
// bm,workspace,pipeline}.cpp of MysteryDove/vapoursynth-LGCR) can be driven
// without VapourSynth. Only tests, the smoke check and the bench's CPU-baseline leg
// load the library built from this file; the product never does.
//
//   oracle_create  restates lgcrCreate          src/plugin.cpp:998-1158
//   oracle_frame   restates lgcrGetFrame        src/plugin.cpp:177-721
//                  with applyFrameChromaSiting  src/plugin.cpp:157-175
//   oracle_sharpen_frame restates sharpenCreate + sharpenGetFrame
//                                               src/plugin.cpp:14-111
//   oracle_trecon_frame  restates tReconCreate + tReconGetFrame
//                                               src/plugin.cpp:723-990
// VapourSynth calls are replaced by plane pointers; the numeric path is the
// reference's, function for function.
#include "lgcr.h"
#include "lgcr_b200.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

using namespace lgcr;

#ifndef ORACLE_TRUE_FLOAT
// The float64 variant force-includes a header that defines this before
// redefining `float`; host I/O keeps the true 32-bit type.
typedef float oracle_f32;
#else
typedef ORACLE_TRUE_FLOAT oracle_f32;
#endif

extern "C" {

typedef struct oracle_debug {
    oracle_f32 *jxx, *jxy, *jyy;   // source luma size
    oracle_f32 *lc, *ms;           // chroma size
    oracle_f32 *plain_u, *plain_v; // output size, base before correction
    uint8_t *seed, *mask;          // source luma size
    uint8_t *chroma_mask;          // chroma size
    uint64_t active_output, active_chroma;
    int has_workset;
} oracle_debug;

} // extern "C"

namespace {

struct OracleFilter {
    LGCRData d;
    lgcr_format fmt{};
};

bool given(int v) { return v != LGCR_UNSET_INT; }
bool given(double v) { return !std::isnan(v); }

void copyError(char *err, size_t len, const char *msg) {
    if (err && len) {
        std::strncpy(err, msg, len - 1);
        err[len - 1] = '\0';
    }
}

// plugin.cpp:157-175
void applyFrameChromaSiting(LGCRData &d, const lgcr_format &fmt, int cl) {
    if (fmt.subsampling_w == 0)
        d.shiftX = 0.0;
    if (fmt.subsampling_h == 0)
        d.shiftY = 0.0;
    if (d.locSet)
        return;
    if (cl < 0)
        return;
    if (fmt.subsampling_w > 0)
        d.shiftX = (cl == 0 || cl == 2 || cl == 4) ? -0.5 : 0.0;
    if (fmt.subsampling_h > 0)
        d.shiftY = (cl == 2 || cl == 3) ? -0.5 : (cl == 4 || cl == 5) ? 0.5 : 0.0;
}

template <class T>
void storePlane(const Plane &src, const lgcr_plane &dst, double scale, double off,
                T lo, T hi) {
    floatToPlane<T>(src, static_cast<uint8_t *>(dst.data), dst.stride, dst.width,
                    dst.height, scale, off, lo, hi);
}

// Float output keeps the 32-bit type even in the float64 variant.
void storeFloatPlane(const Plane &src, const lgcr_plane &dst) {
    for (int y = 0; y < dst.height; ++y) {
        oracle_f32 *row = reinterpret_cast<oracle_f32 *>(
            static_cast<uint8_t *>(dst.data) + dst.stride * y);
        const auto *s = src.row(y);
        for (int x = 0; x < dst.width; ++x)
            row[x] = static_cast<oracle_f32>(s[x]);
    }
}

void copyPlaneOut(const Plane &p, oracle_f32 *dst) {
    if (!dst)
        return;
    for (int y = 0; y < p.h; ++y)
        for (int x = 0; x < p.w; ++x)
            dst[size_t(y) * p.w + x] = static_cast<oracle_f32>(p.row(y)[x]);
}

} // namespace

extern "C" {

// lgcrCreate, plugin.cpp:998-1158
int oracle_create(const lgcr_params *p, const lgcr_format *fmt, void **out,
                  char *err, size_t errlen) {
    auto f = std::make_unique<OracleFilter>();
    LGCRData *d = &f->d;
    f->fmt = *fmt;
    auto fail = [&](const char *msg) {
        copyError(err, errlen, msg);
        return LGCR_E_INVALID;
    };
    const bool isFloat = fmt->sample_type == LGCR_ST_FLOAT;
    if (fmt->color_family != LGCR_CF_YUV || (isFloat && fmt->bits_per_sample != 32) ||
        (!isFloat && (fmt->bits_per_sample < 8 || fmt->bits_per_sample > 16)))
        return fail("LGCR: input must be planar YUV (8-16 bit int or 32 bit float)");
    if (fmt->subsampling_w > 1 || fmt->subsampling_h > 1 ||
        fmt->subsampling_w < 0 || fmt->subsampling_h < 0)
        return fail("LGCR: only 4:4:4 / 4:2:2 / 4:2:0 input is supported");
    if (fmt->width == 0 || fmt->height == 0)
        return fail("LGCR: constant input dimensions required");

    d->outW = given(p->width) ? p->width : fmt->width;
    d->outH = given(p->height) ? p->height : fmt->height;
    if (d->outW <= 0 || d->outH <= 0)
        return fail("LGCR: invalid width/height");

    const std::string k = p->kernel ? p->kernel : "lanczos";
    if (k == "bilinear") {
        d->kernel = Kernel::Bilinear;
        d->support = 1.0;
    } else if (k == "bicubic") {
        d->kernel = Kernel::Bicubic;
        d->support = 2.0;
        d->kp1 = given(p->b) ? p->b : 0.0;
        d->kp2 = given(p->c) ? p->c : 0.6;
    } else if (k == "lanczos") {
        d->kernel = Kernel::Lanczos;
        const long taps = given(p->taps) ? p->taps : 3;
        if (taps < 1 || taps > 64)
            return fail("LGCR: lanczos taps must be in the range 1..64");
        d->kp1 = double(taps);
        d->support = d->kp1;
    } else if (k == "spline16") {
        d->kernel = Kernel::Spline16;
        d->support = 2.0;
    } else if (k == "spline36") {
        d->kernel = Kernel::Spline36;
        d->support = 3.0;
    } else if (k == "jinc") {
        d->kernel = Kernel::Jinc;
        d->radial = true;
        const long taps = given(p->taps) ? p->taps : 3;
        if (taps < 1 || taps > 64)
            return fail("LGCR: jinc taps must be in the range 1..64");
        d->kp1 = double(taps);
        d->support = d->kp1;
        const int n = static_cast<int>(d->support * 1024) + 2;
        d->lut.resize(n);
        for (int i = 0; i < n; ++i)
            d->lut[i] = static_cast<float>(jincWindowed(double(i) / 1024.0, d->support));
        d->lutScale = 1024.0f;
    } else {
        return fail("LGCR: kernel must be \"bilinear\", \"bicubic\", \"lanczos\", "
                    "\"spline16\", \"spline36\" or \"jinc\"");
    }
    d->taps = 2 * static_cast<int>(std::ceil(d->support));

    d->strength = given(p->strength) ? p->strength : 0.8;
    d->sigma = given(p->sigma) ? p->sigma : 0.01;
    d->sratio = given(p->sratio) ? p->sratio : 0.15;
    d->algo = given(p->algo) ? p->algo : 2;
    if (d->algo != 2 && d->algo != 4 && d->algo != 6)
        return fail("LGCR: algo must be 2 (guided), 4 (selector) or 6 (detail transfer)");
    d->sdb = given(p->sdb) ? p->sdb : 3.0;
    d->stretch = given(p->stretch) ? p->stretch : 1.0;
    d->gsigma = given(p->gsigma) ? p->gsigma : 2.5;
    d->rescue = given(p->rescue) ? p->rescue : 1.0;
    d->ridge = given(p->ridge) ? (p->ridge != 0) : true;
    d->cedge = given(p->cedge) ? (p->cedge != 0) : false;
    d->ms = given(p->ms) ? p->ms : 1.0;
    d->qgate = given(p->qgate) ? p->qgate : 1.0;
    d->arMargin = given(p->ar) ? p->ar : 0.0;
    d->reg = given(p->reg) ? p->reg : 0.005;
    if (p->loc) {
        const std::string l = p->loc;
        if (l == "left") d->shiftX = -0.5;
        else if (l == "center") d->shiftX = 0.0;
        else return fail("LGCR: loc must be \"left\" or \"center\"");
        d->locSet = true;
    } else {
        d->shiftX = -0.5;
    }
    d->sparse = given(p->sparse) ? (p->sparse != 0) : true;
    d->bm = given(p->bm) ? (p->bm != 0) : false;
    d->bp = given(p->bp) ? p->bp : 0.0;
    if (fmt->subsampling_w == 0)
        d->shiftX = 0.0;
    if (fmt->subsampling_h == 0)
        d->shiftY = 0.0;
    if (d->strength < 0.0 || d->strength > 1.0 || d->sigma <= 0.0 || d->sratio <= 0.0 ||
        d->sdb <= 0.0 || d->stretch < 0.0 || d->gsigma <= 0.0 || d->reg <= 0.0 ||
        d->bp < 0.0 || d->bp > 1.0 || d->ms < 0.0 || d->ms > 1.0 ||
        d->qgate < 0.0 || d->qgate > 1.0 || d->rescue < 0.0 || d->rescue > 1.0)
        return fail("LGCR: invalid parameter range (need 0<=strength/rescue<=1, "
                    "0<=bp/ms/qgate<=1, sigma/sratio/sdb/gsigma/reg>0, stretch>=0)");
    *out = f.release();
    return LGCR_OK;
}

void oracle_destroy(void *handle) { delete static_cast<OracleFilter *>(handle); }

// lgcrGetFrame, plugin.cpp:177-721. `threads` sizes the workspace pool like
// coreInfo.numThreads; `profile` turns on PipelineMetrics (counters only).
int oracle_frame(void *handle, const lgcr_plane in[3], const lgcr_plane out[3],
                 int chroma_location, int threads, int profile,
                 oracle_debug *dbg, lgcr_frame_stats *stats) {
    OracleFilter *filter = static_cast<OracleFilter *>(handle);
    const lgcr_format &fmt = filter->fmt;
    PipelineMetrics frameMetrics;
    PipelineMetrics *metrics = profile ? &frameMetrics : nullptr;

    LGCRData dloc = filter->d;
    applyFrameChromaSiting(dloc, fmt, chroma_location);
    const LGCRData *d = &dloc;

    const int sw = in[0].width, sh = in[0].height;
    const int cw = in[1].width, ch = in[1].height;
    const bool isFloat = fmt.sample_type == LGCR_ST_FLOAT;
    const int bytesPerSample = isFloat ? 4 : (fmt.bits_per_sample > 8 ? 2 : 1);
    const double yScale = isFloat ? 1.0 : 1.0 / double((1 << fmt.bits_per_sample) - 1);
    const double cOffset = isFloat ? 0.0 : -0.5;

    FrameWorkspaceLease workspaceLease = d->workspacePool->acquire(threads);
    FrameWorkspace &workspace = workspaceLease.get();
    Plane *sourceY = &workspace.sourceY;
    Plane *sourceU = &workspace.sourceU;
    Plane *sourceV = &workspace.sourceV;
    // Float input: the reference borrows the frame as zero-copy views; the
    // values are identical to converting with scale 1 and offset 0.
    workspace.sourceY.resizeDiscard(sw, sh);
    workspace.sourceU.resizeDiscard(cw, ch);
    workspace.sourceV.resizeDiscard(cw, ch);
    const uint8_t *src0 = static_cast<const uint8_t *>(in[0].data);
    const uint8_t *src1 = static_cast<const uint8_t *>(in[1].data);
    const uint8_t *src2 = static_cast<const uint8_t *>(in[2].data);
    if (isFloat) {
        const uint8_t *srcs[3] = { src0, src1, src2 };
        Plane *dsts[3] = { sourceY, sourceU, sourceV };
        for (int p = 0; p < 3; ++p)
            for (int row = 0; row < dsts[p]->h; ++row) {
                const oracle_f32 *s = reinterpret_cast<const oracle_f32 *>(
                    srcs[p] + in[p].stride * row);
                auto *t = dsts[p]->row(row);
                for (int x = 0; x < dsts[p]->w; ++x)
                    t[x] = s[x];
            }
    } else if (bytesPerSample == 1) {
        planeToFloat<uint8_t>(src0, in[0].stride, *sourceY, sw, sh, yScale, 0.0);
        planeToFloat<uint8_t>(src1, in[1].stride, *sourceU, cw, ch, yScale, cOffset);
        planeToFloat<uint8_t>(src2, in[2].stride, *sourceV, cw, ch, yScale, cOffset);
    } else {
        planeToFloat<uint16_t>(src0, in[0].stride, *sourceY, sw, sh, yScale, 0.0);
        planeToFloat<uint16_t>(src1, in[1].stride, *sourceU, cw, ch, yScale, cOffset);
        planeToFloat<uint16_t>(src2, in[2].stride, *sourceV, cw, ch, yScale, cOffset);
    }
    Plane &y = *sourceY;
    Plane &cb = *sourceU;
    Plane &cr = *sourceV;

    const double rw = double(sw) / cw;
    const double rh = double(sh) / ch;
    const bool sameSize = d->outW == sw && d->outH == sh;
    const double outScaleY = isFloat ? 1.0 : double((1 << fmt.bits_per_sample) - 1);
    const int maxCode = (1 << fmt.bits_per_sample) - 1;

    // Luma (plugin.cpp:273-316). Same size: the source plane is shared.
    if (sameSize) {
        if (out[0].data)
            for (int row = 0; row < sh; ++row)
                std::memcpy(static_cast<uint8_t *>(out[0].data) + out[0].stride * row,
                            src0 + in[0].stride * row, size_t(sw) * bytesPerSample);
    } else {
        workspace.fullSlot0.resizeDiscard(d->outW, d->outH);
        Plane *outputY = &workspace.fullSlot0;
        if (d->radial) {
            resampleRadial(y, *outputY, *d);
        } else {
            const auto th = cachedWeights(d, sw, d->outW, 0.0);
            const auto tv = cachedWeights(d, sh, d->outH, 0.0);
            workspace.fullSlot1.resizeDiscard(d->outW, sh);
            resampleH(y, workspace.fullSlot1, *th);
            resampleV(workspace.fullSlot1, *outputY, *tv);
        }
        if (isFloat)
            storeFloatPlane(*outputY, out[0]);
        else if (bytesPerSample == 1)
            storePlane<uint8_t>(*outputY, out[0], outScaleY, 0.0, 0, 255);
        else
            storePlane<uint16_t>(*outputY, out[0], outScaleY, 0.0, 0, uint16_t(maxCode));
    }

    GuideMaps gm;
    SparseWorkset sparseWorkset;
    bool hasSparseWorkset = false;
    std::shared_ptr<const ChromaAxis> frameAxisX, frameAxisY;
    uint64_t sparseActive = 0, sparseTotal = 0;
    if (d->strength > 0.0) {
        const double trustThreshold = d->algo == 4 ? 0.25 * d->sigma : d->sigma;
        gm = buildGuideMaps(y, y, cw, ch, rw, rh, d->shiftX, d->shiftY,
                            metrics, d->sparse ? trustThreshold : -1.0,
                            &workspace.scratch);
        if (dbg) {
            copyPlaneOut(gm.jxx, dbg->jxx);
            copyPlaneOut(gm.jxy, dbg->jxy);
            copyPlaneOut(gm.jyy, dbg->jyy);
            copyPlaneOut(gm.lc, dbg->lc);
            if (dbg->seed && !gm.trustSeed.empty())
                std::memcpy(dbg->seed, gm.trustSeed.data(), gm.trustSeed.size());
        }
        if (d->sparse) {
            const int dil = int(std::ceil(d->support * std::max(rw, rh))) + 8;
            std::vector<uint8_t> trustMask = buildTrustMask(gm, sw, sh, trustThreshold, dil, metrics);
            sparseTotal = trustMask.size();
            sparseActive = static_cast<uint64_t>(
                std::count(trustMask.begin(), trustMask.end(), uint8_t{1}));
            if (dbg && dbg->mask)
                std::memcpy(dbg->mask, trustMask.data(), trustMask.size());
            frameAxisX = cachedChromaAxis(d, sw, d->outW, rw, d->shiftX);
            frameAxisY = cachedChromaAxis(d, sh, d->outH, rh, d->shiftY);
            sparseWorkset = buildSparseWorkset(std::move(trustMask), sw, sh, d->outW,
                                               d->outH, *frameAxisX, *frameAxisY, cw, ch);
            hasSparseWorkset = true;
            if (dbg) {
                if (dbg->chroma_mask)
                    std::memcpy(dbg->chroma_mask, sparseWorkset.chromaMask.data(),
                                sparseWorkset.chromaMask.size());
                dbg->active_output = sparseWorkset.activeOutputPixels;
                dbg->active_chroma = sparseWorkset.activeChromaPixels;
                dbg->has_workset = 1;
            }
        }
        if (d->ms > 0.0) {
            gm.ms = buildMutualGate(gm.lc, cb, cr, d->sigma,
                                    hasSparseWorkset ? sparseWorkset.chromaMask.data() : nullptr,
                                    cw, hasSparseWorkset ? &sparseWorkset : nullptr,
                                    metrics, &workspace.scratch);
            if (dbg)
                copyPlaneOut(gm.ms, dbg->ms);
        }
    }

    const bool needsBackProjection = d->bp > 0.0 && d->outW == sw &&
        d->outH == sh && cw * 2 == sw && ch * 2 == sh;
    workspace.fullSlot0.resizeDiscard(d->outW, d->outH);
    workspace.fullSlot1.resizeDiscard(d->outW, d->outH);
    Plane &cOutU = workspace.fullSlot0;
    Plane &cOutV = workspace.fullSlot1;
    auto capturePlain = [&]() {
        if (dbg) {
            copyPlaneOut(cOutU, dbg->plain_u);
            copyPlaneOut(cOutV, dbg->plain_v);
        }
    };
    if (d->algo == 4) {
        plainChroma(d, cb, cr, y, gm, sw, sh, cw, ch, cOutU, cOutV, metrics);
        capturePlain();
        if (d->strength > 0.0) {
            if (!isFloat) {
                LGFMaps lgf = buildLGFMaps(d, y, cb, cr, cw, ch, rw, rh, metrics,
                                           nullptr, 0, &workspace.scratch);
                if (gm.ms.w > 0)
                    for (int j = 0; j < ch; ++j)
                        for (int i = 0; i < cw; ++i) {
                            const float f = 1.0f - float(d->ms) * (1.0f - gm.ms.at(i, j));
                            lgf.confU.at(i, j) *= f;
                            lgf.confV.at(i, j) *= f;
                        }
                LGCRData integerSelector = *d;
                integerSelector.algo = 2;
                integerSelector.strength = 1.0;
                ChromaJob job;
                job.srcU = &cb; job.srcV = &cr; job.srcY = &y; job.gm = &gm;
                job.dstU = &cOutU; job.dstV = &cOutV;
                job.srcLumaW = sw; job.srcLumaH = sh;
                job.rw = rw; job.rh = rh;
                job.shiftX = d->shiftX; job.shiftY = d->shiftY;
                job.d = &integerSelector;
                job.selectorMaps = &lgf;
                job.selectorStrength = float(d->strength);
                job.plainU = &cOutU;
                job.plainV = &cOutV;
                job.metrics = metrics;
                if (hasSparseWorkset)
                    job.workset = &sparseWorkset;
                reconstructChroma(job);
            } else {
                LGCRData d4 = *d;
                d4.algo = 2;
                d4.strength = 1.0;
                const bool compressedSelector = hasSparseWorkset &&
                    !sparseWorkset.outputDenseFallback();
                Plane guidedU, guidedV, w2, w3;
                CompressedSelector selector;
                if (compressedSelector)
                    selector.resize(sparseWorkset.activeOutputPixels);
                else {
                    guidedU = Plane(d->outW, d->outH);
                    guidedV = Plane(d->outW, d->outH);
                    w2 = Plane(d->outW, d->outH);
                    w3 = Plane(d->outW, d->outH);
                }
                ChromaJob job;
                job.srcU = &cb; job.srcV = &cr; job.srcY = &y; job.gm = &gm;
                job.dstU = compressedSelector ? &cOutU : &guidedU;
                job.dstV = compressedSelector ? &cOutV : &guidedV;
                job.srcLumaW = sw; job.srcLumaH = sh;
                job.rw = rw; job.rh = rh; job.shiftX = d->shiftX; job.shiftY = d->shiftY;
                job.d = &d4;
                job.selectorStrength = float(d->strength);
                job.selectorMetadata = true;
                if (compressedSelector) {
                    job.compressedSelector = &selector;
                    job.plainU = &cOutU;
                    job.plainV = &cOutV;
                } else {
                    job.selectorW2 = &w2;
                    job.selectorW3 = &w3;
                }
                job.metrics = metrics;
                if (hasSparseWorkset)
                    job.workset = &sparseWorkset;
                reconstructChroma(job);

                const auto ax = frameAxisX ? frameAxisX
                    : cachedChromaAxis(d, sw, d->outW, rw, d->shiftX);
                const auto ay = frameAxisY ? frameAxisY
                    : cachedChromaAxis(d, sh, d->outH, rh, d->shiftY);
                std::vector<uint8_t> roi(size_t(cw) * ch, 0);
                auto markRoi = [&](int ox, int oy, float selectorW3) {
                    if (selectorW3 < 1e-4f)
                        return;
                    const int cx0 = ax->chromaBilin.i0[ox];
                    const int cx1 = std::min(cx0 + 1, cw - 1);
                    const int cy0 = ay->chromaBilin.i0[oy];
                    const int cy1 = std::min(cy0 + 1, ch - 1);
                    roi[size_t(cy0) * cw + cx0] = 1;
                    roi[size_t(cy0) * cw + cx1] = 1;
                    roi[size_t(cy1) * cw + cx0] = 1;
                    roi[size_t(cy1) * cw + cx1] = 1;
                };
                if (compressedSelector) {
                    for (int oy = 0; oy < d->outH; ++oy) {
                        size_t index = sparseWorkset.outputIndexRowOffsets[oy];
                        for (size_t s = sparseWorkset.outputRowOffsets[oy];
                             s < sparseWorkset.outputRowOffsets[oy + 1]; ++s) {
                            const SparseSpan span = sparseWorkset.outputSpans[s];
                            for (int ox = span.begin; ox < span.end; ++ox, ++index)
                                markRoi(ox, oy, selector.w3[index]);
                        }
                    }
                } else if (hasSparseWorkset) {
                    for (int oy = 0; oy < d->outH; ++oy)
                        for (size_t s = sparseWorkset.outputRowOffsets[oy];
                             s < sparseWorkset.outputRowOffsets[oy + 1]; ++s) {
                            const SparseSpan span = sparseWorkset.outputSpans[s];
                            for (int ox = span.begin; ox < span.end; ++ox)
                                markRoi(ox, oy, w3.row(oy)[ox]);
                        }
                } else {
                    for (int oy = 0; oy < d->outH; ++oy)
                        for (int ox = 0; ox < d->outW; ++ox)
                            markRoi(ox, oy, w3.row(oy)[ox]);
                }
                LGFMaps lgf = buildLGFMaps(d, y, cb, cr, cw, ch, rw, rh, metrics,
                                           roi.data(), cw, &workspace.scratch);
                if (gm.ms.w > 0)
                    for (int j = 0; j < ch; ++j)
                        for (int i = 0; i < cw; ++i) {
                            if (roi[size_t(j) * cw + i] == 0)
                                continue;
                            const float f = 1.0f - float(d->ms) * (1.0f - gm.ms.at(i, j));
                            lgf.confU.at(i, j) *= f;
                            lgf.confV.at(i, j) *= f;
                        }
                if (compressedSelector)
                    blendSelectorCompressed(cOutU, cOutV, selector, lgf.aU, lgf.bU, lgf.aV,
                                            lgf.bV, lgf.confU, lgf.confV, y, *ax, *ay,
                                            sparseWorkset, float(d->strength), metrics);
                else
                    blendSelector(cOutU, cOutV, guidedU, guidedV, lgf.aU, lgf.bU, lgf.aV,
                                  lgf.bV, lgf.confU, lgf.confV, y, *ax, *ay, w2, w3, cw, ch,
                                  float(d->strength),
                                  hasSparseWorkset ? &sparseWorkset : nullptr, metrics);
            }
        }
    } else if (d->algo == 6) {
        plainChroma(d, cb, cr, y, gm, sw, sh, cw, ch, cOutU, cOutV, metrics);
        capturePlain();
        if (d->strength > 0.0) {
            AffineMaps af = buildAffineMaps(d, y, cb, cr, cw, ch, rw, rh, metrics, &gm,
                                            hasSparseWorkset ? &sparseWorkset : nullptr,
                                            &workspace.scratch);
            gm.lc = Plane();
            buildDetailMap(d, y, cw, ch, rw, rh, af, metrics);
            const auto ax = frameAxisX ? frameAxisX
                : cachedChromaAxis(d, sw, d->outW, rw, d->shiftX);
            const auto ay = frameAxisY ? frameAxisY
                : cachedChromaAxis(d, sh, d->outH, rh, d->shiftY);
            const uint8_t *mp = nullptr;
            int mw = 0, mh = 0;
            if (hasSparseWorkset) {
                mp = sparseWorkset.mask.data();
                mw = sw;
                mh = sh;
            }
            detailTransfer(d, cOutU, cOutV, af, gm, *ax, *ay, mp, mw, mh,
                           hasSparseWorkset ? &sparseWorkset : nullptr, metrics);
        }
    } else if (d->strength == 0.0) {
        plainChroma(d, cb, cr, y, gm, sw, sh, cw, ch, cOutU, cOutV, metrics);
        capturePlain();
    } else {
        CompressedChromaHull plainHull;
        const bool reusePlainHull = hasSparseWorkset &&
            !sparseWorkset.outputDenseFallback() && !d->radial &&
            d->kernel != Kernel::Bilinear;
        if (hasSparseWorkset) {
            if (reusePlainHull)
                plainHull.resize(sparseWorkset.activeOutputPixels);
            plainChroma(d, cb, cr, y, gm, sw, sh, cw, ch, cOutU, cOutV, metrics,
                        reusePlainHull ? &plainHull : nullptr,
                        reusePlainHull ? &sparseWorkset : nullptr);
            capturePlain();
        }
        ChromaJob job;
        job.srcU = &cb;
        job.srcV = &cr;
        job.srcY = &y;
        job.gm = &gm;
        job.dstU = &cOutU;
        job.dstV = &cOutV;
        job.srcLumaW = sw;
        job.srcLumaH = sh;
        job.rw = rw;
        job.rh = rh;
        job.shiftX = d->shiftX;
        job.shiftY = d->shiftY;
        job.d = d;
        job.metrics = metrics;
        if (hasSparseWorkset) {
            job.workset = &sparseWorkset;
            job.plainU = &cOutU;
            job.plainV = &cOutV;
            if (reusePlainHull)
                job.plainHull = &plainHull;
        }
        reconstructChroma(job);
    }
    if (d->bm)
        collaborativeChromaFilter(y, cOutU, cOutV, float(d->sigma), metrics);
    if (needsBackProjection) {
        backProject(cOutU, cb, float(d->bp));
        backProject(cOutV, cr, float(d->bp));
    }

    for (int p = 0; p < 2; ++p) {
        const Plane &cOut = (p == 0) ? cOutU : cOutV;
        const double outScale = isFloat ? 1.0 : double((1 << fmt.bits_per_sample) - 1);
        const double outOffset = isFloat ? 0.0 : 0.5 * outScale;
        if (isFloat)
            storeFloatPlane(cOut, out[p + 1]);
        else if (bytesPerSample == 1)
            storePlane<uint8_t>(cOut, out[p + 1], outScale, outOffset, 0, 255);
        else
            storePlane<uint16_t>(cOut, out[p + 1], outScale, outOffset, 0, uint16_t(maxCode));
    }

    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->output_pixels = uint64_t(d->outW) * d->outH;
        stats->sparse_active_pixels = sparseActive;
        stats->sparse_total_pixels = sparseTotal;
        stats->active_output_pixels = hasSparseWorkset ? sparseWorkset.activeOutputPixels
                                                       : stats->output_pixels;
        stats->active_chroma_pixels = hasSparseWorkset ? sparseWorkset.activeChromaPixels
                                                       : uint64_t(cw) * ch;
        stats->sparse_active_ratio = sparseTotal ? double(sparseActive) / sparseTotal : 1.0;
    }
    return LGCR_OK;
}

// Reference geometry tables, for pinning the host-side restatement.
// kernels.cpp:337-404 (buildChromaAxisUncached via cachedChromaAxis).
int oracle_chroma_axis(void *handle, int srcLumaN, int dstLumaN, double r, double sitShift,
                       int *start, oracle_f32 *w, oracle_f32 *am, oracle_f32 *pos,
                       oracle_f32 *lpos, int *cbI0, oracle_f32 *cbF, int *lbI0,
                       oracle_f32 *lbF, int *supOut) {
    OracleFilter *filter = static_cast<OracleFilter *>(handle);
    const auto ax = cachedChromaAxis(&filter->d, srcLumaN, dstLumaN, r, sitShift);
    *supOut = ax->sup;
    for (int i = 0; i < ax->n; ++i) {
        if (start) start[i] = ax->start[i];
        if (pos) pos[i] = ax->pos[i];
        if (lpos) lpos[i] = ax->lpos[i];
        if (cbI0) cbI0[i] = ax->chromaBilin.i0[i];
        if (cbF) cbF[i] = ax->chromaBilin.f[i];
        if (lbI0) lbI0[i] = ax->lumaBilin.i0[i];
        if (lbF) lbF[i] = ax->lumaBilin.f[i];
        for (int j = 0; j < ax->sup; ++j) {
            if (w) w[size_t(i) * ax->sup + j] = ax->w[size_t(i) * ax->sup + j];
            if (am) am[size_t(i) * ax->sup + j] = ax->am[size_t(i) * ax->sup + j];
        }
    }
    return LGCR_OK;
}

// kernels.cpp:135-167
int oracle_weights(void *handle, int srcN, int dstN, double shift, int *start,
                   oracle_f32 *w, int *supOut) {
    OracleFilter *filter = static_cast<OracleFilter *>(handle);
    const auto t = cachedWeights(&filter->d, srcN, dstN, shift);
    *supOut = t->sup;
    if (start)
        for (int i = 0; i < t->n; ++i)
            start[i] = t->start[i];
    if (w)
        for (size_t i = 0; i < t->w.size(); ++i)
            w[i] = t->w[i];
    return LGCR_OK;
}

// plugin.cpp:1071-1076
int oracle_jinc_lut(void *handle, oracle_f32 *lut, int *n) {
    OracleFilter *filter = static_cast<OracleFilter *>(handle);
    *n = int(filter->d.lut.size());
    if (lut)
        for (size_t i = 0; i < filter->d.lut.size(); ++i)
            lut[i] = filter->d.lut[i];
    return LGCR_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Sharpen (plugin.cpp:14-111): sharpenCreate's argument defaults and checks,
// then sharpenGetFrame's sequence over raw planes, calling the reference's
// planeToFloat, sharpenPlane (algos.cpp:595-659), buildGuideMaps and
// floatToPlane.
// ---------------------------------------------------------------------------
namespace {

void extractPlanes(const lgcr_plane *in, const lgcr_format &fmt, Plane &y, Plane &cb, Plane &cr,
                   bool chromaOffset) {
    const bool isFloat = fmt.sample_type == LGCR_ST_FLOAT;
    const int bytes = isFloat ? 4 : (fmt.bits_per_sample > 8 ? 2 : 1);
    const double yScale = isFloat ? 1.0 : 1.0 / double((1 << fmt.bits_per_sample) - 1);
    Plane *dst[3] = { &y, &cb, &cr };
    for (int p = 0; p < 3; ++p) {
        const uint8_t *src = static_cast<const uint8_t *>(in[p].data);
        const double off = (p == 0 || isFloat || !chromaOffset) ? 0.0 : -0.5;
        if (isFloat) {
            // planeToFloat<float>(.., 1.0, 0.0): s * 1.0 + 0.0 in double
            for (int row = 0; row < dst[p]->h; ++row) {
                const oracle_f32 *s = reinterpret_cast<const oracle_f32 *>(src + in[p].stride * row);
                for (int x = 0; x < dst[p]->w; ++x)
                    dst[p]->row(row)[x] = static_cast<oracle_f32>(s[x] * 1.0 + 0.0);
            }
        } else if (bytes == 1) {
            planeToFloat<uint8_t>(src, in[p].stride, *dst[p], dst[p]->w, dst[p]->h, yScale, off);
        } else {
            planeToFloat<uint16_t>(src, in[p].stride, *dst[p], dst[p]->w, dst[p]->h, yScale, off);
        }
    }
}

void storeOutputPlane(const Plane &s, const lgcr_plane &out, const lgcr_format &fmt, bool chroma) {
    const bool isFloat = fmt.sample_type == LGCR_ST_FLOAT;
    const int bytes = isFloat ? 4 : (fmt.bits_per_sample > 8 ? 2 : 1);
    const double outScale = isFloat ? 1.0 : double((1 << fmt.bits_per_sample) - 1);
    const double outOff = (!chroma || isFloat) ? 0.0 : 0.5 * outScale;
    if (isFloat)
        storeFloatPlane(s, out);
    else if (bytes == 1)
        storePlane<uint8_t>(s, out, outScale, outOff, 0, 255);
    else
        storePlane<uint16_t>(s, out, outScale, outOff, 0,
                             uint16_t((1 << fmt.bits_per_sample) - 1));
}

} // namespace

extern "C" int oracle_sharpen_frame(const lgcr_format *fmt, double alpha, double sigma,
                                    double sratio, double gspatial, double ar,
                                    const lgcr_plane *in, const lgcr_plane *out, char *err,
                                    size_t errlen) {
    if (fmt->color_family != LGCR_CF_YUV ||
        (fmt->sample_type == LGCR_ST_FLOAT && fmt->bits_per_sample != 32)) {
        copyError(err, errlen, "LGCR Sharpen: planar YUV only");
        return LGCR_E_INVALID;
    }
    SharpenData d;
    if (given(alpha)) d.alpha = alpha;
    if (given(sigma)) d.sigma = sigma;
    if (given(sratio)) d.sratio = sratio;
    if (given(gspatial)) d.gspatial = gspatial;
    if (given(ar)) d.arMargin = ar;
    if (d.sigma <= 0.0 || d.sratio <= 0.0 || d.gspatial <= 0.0) {
        copyError(err, errlen, "LGCR Sharpen: sigma/sratio/gspatial must be > 0");
        return LGCR_E_INVALID;
    }
    const int sw = in[0].width, sh = in[0].height, cw = in[1].width, ch = in[1].height;
    Plane y(sw, sh), cb(cw, ch), cr(cw, ch);
    extractPlanes(in, *fmt, y, cb, cr, true);
    sharpenPlane(y, nullptr, y, 1.0, 1.0, 0.0, 0.0, d);
    if (cw != sw || ch != sh) {
        const double rw = double(sw) / cw, rh = double(sh) / ch;
        GuideMaps gm = buildGuideMaps(y, y, cw, ch, rw, rh, -0.5, 0.0);
        sharpenPlane(cb, &gm.lc, y, rw, rh, -0.5, 0.0, d);
        sharpenPlane(cr, &gm.lc, y, rw, rh, -0.5, 0.0, d);
    } else {
        sharpenPlane(cb, nullptr, cb, 1.0, 1.0, 0.0, 0.0, d);
        sharpenPlane(cr, nullptr, cr, 1.0, 1.0, 0.0, 0.0, d);
    }
    storeOutputPlane(y, out[0], *fmt, false);
    storeOutputPlane(cb, out[1], *fmt, true);
    storeOutputPlane(cr, out[2], *fmt, true);
    return LGCR_OK;
}

// ---------------------------------------------------------------------------
// TRecon (plugin.cpp:723-990): tReconCreate's defaults and checks, then
// tReconGetFrame's sequence over raw planes -- per neighbour the reference's
// blockMatch and applyChromaConsistency (algos.cpp:683-807) and buildLcMap,
// then guide maps, mutual gate, optional trust mask + plain base, and
// reconstructChroma with the temporal taps (recon.cpp:642-745), optional
// collaborativeChromaFilter, output conversion.
// ---------------------------------------------------------------------------
namespace {

int tReconSetup(const lgcr_trecon_params *p, const lgcr_format *fmt, int numFrames,
                LGCRData &d, char *err, size_t errlen) {
    auto fail = [&](const char *msg) {
        copyError(err, errlen, msg);
        return LGCR_E_INVALID;
    };
    const bool isFloat = fmt->sample_type == LGCR_ST_FLOAT;
    if (fmt->color_family != LGCR_CF_YUV || (isFloat && fmt->bits_per_sample != 32) ||
        (!isFloat && (fmt->bits_per_sample < 8 || fmt->bits_per_sample > 16)) ||
        fmt->subsampling_w > 1 || fmt->subsampling_h > 1 || fmt->subsampling_w < 0 ||
        fmt->subsampling_h < 0)
        return fail("TRecon: planar YUV 444/422/420, 8-16 bit int or 32 bit float");
    if (fmt->width == 0 || fmt->height == 0 || numFrames == 0)
        return fail("TRecon: constant dimensions and frame count required");
    d.outW = fmt->width;
    d.outH = fmt->height;
    d.strength = given(p->strength) ? p->strength : 0.8;
    d.sigma = given(p->sigma) ? p->sigma : 0.01;
    d.sratio = given(p->sratio) ? p->sratio : 0.15;
    d.sdb = given(p->sdb) ? p->sdb : 3.0;
    d.gsigma = given(p->gsigma) ? p->gsigma : 2.5;
    d.stretch = given(p->stretch) ? p->stretch : 1.0;
    d.arMargin = given(p->ar) ? p->ar : 0.0;
    d.ms = given(p->ms) ? p->ms : 1.0;
    d.trad = given(p->trad) ? p->trad : 1;
    d.tsearch = given(p->tsearch) ? p->tsearch : 6;
    d.tsad = given(p->tsad) ? p->tsad : 0.02;
    if (d.strength < 0.0 || d.strength > 1.0 || d.sigma <= 0.0 || d.sratio <= 0.0 ||
        d.sdb <= 0.0 || d.stretch < 0.0 || d.gsigma <= 0.0 || d.ms < 0.0 || d.ms > 1.0 ||
        d.trad < 0 || d.trad > 8 || d.tsearch < 0 || d.tsearch > 64 || d.tsad <= 0.0)
        return fail("TRecon: invalid parameter range (need 0<=strength<=1, "
                    "sigma/sratio/sdb/gsigma/tsad>0, stretch>=0, 0<=trad<=8, 0<=tsearch<=64)");
    d.ridge = given(p->ridge) ? (p->ridge != 0) : true;
    d.bm = given(p->bm) ? (p->bm != 0) : false;
    d.sparse = given(p->sparse) ? (p->sparse != 0) : false;
    d.algo = 2;
    d.taps = 2 * 3;
    d.support = 3.0;
    d.kernel = Kernel::Lanczos;
    return LGCR_OK;
}

} // namespace

extern "C" int oracle_trecon_frame(const lgcr_trecon_params *p, const lgcr_format *fmt,
                                   int numFrames, const lgcr_plane *cur, const lgcr_plane *nbrPlanes,
                                   int count, const lgcr_plane *out, int chroma_location,
                                   char *err, size_t errlen) {
    LGCRData dbase;
    const int status = tReconSetup(p, fmt, numFrames, dbase, err, errlen);
    if (status != LGCR_OK)
        return status;
    LGCRData dloc = dbase;
    applyFrameChromaSiting(dloc, *fmt, chroma_location);
    const LGCRData *d = &dloc;
    const int sw = cur[0].width, sh = cur[0].height, cw = cur[1].width, ch = cur[1].height;
    const double rw = double(sw) / cw, rh = double(sh) / ch;
    Plane y(sw, sh), cb(cw, ch), cr(cw, ch);
    extractPlanes(cur, *fmt, y, cb, cr, true);

    std::vector<TemporalNbr> nbrs;
    std::vector<std::unique_ptr<Plane>> store;
    std::vector<std::vector<int16_t>> mvStoreX, mvStoreY;
    std::vector<std::vector<float>> confStore;
    nbrs.reserve(count);
    mvStoreX.reserve(count);
    mvStoreY.reserve(count);
    confStore.reserve(count);
    if (d->strength > 0.0) {
        for (int k = 0; k < count; ++k) {
            auto ny = std::make_unique<Plane>(sw, sh);
            auto nu = std::make_unique<Plane>(cw, ch);
            auto nv = std::make_unique<Plane>(cw, ch);
            extractPlanes(nbrPlanes + 3 * k, *fmt, *ny, *nu, *nv, true);
            mvStoreX.emplace_back();
            mvStoreY.emplace_back();
            confStore.emplace_back();
            int bw = 0, bh = 0;
            blockMatch(y, *ny, 16, d->tsearch, float(d->tsad), mvStoreX.back(), mvStoreY.back(),
                       confStore.back(), bw, bh);
            applyChromaConsistency(cb, cr, *nu, *nv, sw, sh, 16, mvStoreX.back(),
                                   mvStoreY.back(), bw, bh, confStore.back());
            auto lc = std::make_unique<Plane>(buildLcMap(*ny, cw, ch, rw, rh, d->shiftX, d->shiftY));
            TemporalNbr nb;
            nb.U = nu.get();
            nb.V = nv.get();
            nb.lc = lc.get();
            nb.mvx = &mvStoreX.back();
            nb.mvy = &mvStoreY.back();
            nb.tconf = &confStore.back();
            nb.bw = bw;
            nb.bh = bh;
            nb.block = 16;
            nbrs.push_back(nb);
            store.push_back(std::move(ny));
            store.push_back(std::move(nu));
            store.push_back(std::move(nv));
            store.push_back(std::move(lc));
        }
    }
    GuideMaps gm;
    if (d->strength > 0.0) {
        gm = buildGuideMaps(y, y, cw, ch, rw, rh, d->shiftX, d->shiftY);
        if (d->ms > 0.0)
            gm.ms = buildMutualGate(gm.lc, cb, cr, d->sigma);
    }
    storeOutputPlane(y, out[0], *fmt, false);

    Plane cOutU(sw, sh), cOutV(sw, sh);
    std::vector<uint8_t> mask;
    if (d->sparse && d->strength > 0.0) {
        const int dil = int(std::ceil(d->support * std::max(rw, rh))) + 8;
        mask = buildTrustMask(gm, sw, sh, d->sigma, dil);
        plainChroma(d, cb, cr, y, gm, sw, sh, cw, ch, cOutU, cOutV);
    }
    {
        ChromaJob job;
        job.srcU = &cb;
        job.srcV = &cr;
        job.srcY = &y;
        job.gm = &gm;
        job.dstU = &cOutU;
        job.dstV = &cOutV;
        job.srcLumaW = sw;
        job.srcLumaH = sh;
        job.rw = rw;
        job.rh = rh;
        job.shiftX = d->shiftX;
        job.shiftY = d->shiftY;
        job.d = d;
        if (!mask.empty()) {
            job.mask = mask.data();
            job.maskW = sw;
            job.maskH = sh;
            job.plainU = &cOutU;
            job.plainV = &cOutV;
        }
        if (!nbrs.empty())
            job.nbrs = &nbrs;
        reconstructChroma(job);
    }
    if (d->bm)
        collaborativeChromaFilter(y, cOutU, cOutV, float(d->sigma));
    storeOutputPlane(cOutU, out[1], *fmt, true);
    storeOutputPlane(cOutV, out[2], *fmt, true);
    return LGCR_OK;
}
