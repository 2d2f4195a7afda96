// Host runtime: filter creation (lgcrCreate, src/plugin.cpp:998-1158),
// per-siting resident tables, workspaces and the stage scheduler that
// replaces lgcrGetFrame's sequence of stage calls (src/plugin.cpp:177-721)
// with one launch per stage covering every frame of a batch.
#include "impl.h"
#include "kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace lgcr_b200 {

static thread_local std::string tlsError;

const char *setError(const std::string &msg) {
    tlsError = msg;
    return tlsError.c_str();
}

const char *lastError() { return tlsError.c_str(); }

int cudaFail(cudaError_t e, const char *where) {
    setError(std::string("LGCR: CUDA error in ") + where + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? LGCR_E_NOMEM : LGCR_E_CUDA;
}

DeviceArena::~DeviceArena() {
    if (base_)
        cudaFree(base_);
}

bool DeviceArena::commit() {
    if (base_ || size_ == 0)
        return true;
    return cudaMalloc(&base_, size_) == cudaSuccess;
}

Workspace::~Workspace() {
    if (done)
        cudaEventDestroy(done);
    for (int i = 0; i < 3; ++i) {
        if (pinnedIn[i])
            cudaFreeHost(pinnedIn[i]);
        if (pinnedOut[i])
            cudaFreeHost(pinnedOut[i]);
    }
    if (hJob)
        cudaFreeHost(hJob);
}

Filter::~Filter() {
    if (dLut)
        cudaFree(dLut);
}

// ---------------------------------------------------------------------------
// lgcrCreate
// ---------------------------------------------------------------------------
static bool given(int v) { return v != LGCR_UNSET_INT; }
static bool given(double v) { return !std::isnan(v); }

int createFilter(const lgcr_params *pp, const lgcr_format *fmt, Filter **out, std::string &err) {
    auto fail = [&](const char *msg) { err = msg; return LGCR_E_INVALID; };
    if (!pp || !fmt || !out)
        return fail("LGCR: null argument");
    const lgcr_params &a = *pp;
    const bool isFloat = fmt->sample_type == LGCR_ST_FLOAT;
    if (fmt->color_family != LGCR_CF_YUV || (isFloat && fmt->bits_per_sample != 32) ||
        (!isFloat && (fmt->bits_per_sample < 8 || fmt->bits_per_sample > 16)) ||
        (fmt->sample_type != LGCR_ST_FLOAT && fmt->sample_type != LGCR_ST_INTEGER))
        return fail("LGCR: input must be planar YUV (8-16 bit int or 32 bit float)");
    if (fmt->subsampling_w > 1 || fmt->subsampling_h > 1 || fmt->subsampling_w < 0 ||
        fmt->subsampling_h < 0)
        return fail("LGCR: only 4:4:4 / 4:2:2 / 4:2:0 input is supported");
    if (fmt->width <= 0 || fmt->height <= 0)
        return fail("LGCR: constant input dimensions required");

    auto f = std::make_unique<Filter>();
    FilterParams &d = f->p;
    f->fmt = *fmt;
    d.outW = given(a.width) ? a.width : fmt->width;
    d.outH = given(a.height) ? a.height : fmt->height;
    if (d.outW <= 0 || d.outH <= 0)
        return fail("LGCR: invalid width/height");

    const std::string k = a.kernel ? a.kernel : "lanczos";
    KernelSpec &ks = d.k;
    if (k == "bilinear") {
        ks.kernel = Kernel::Bilinear;
        ks.support = 1.0;
    } else if (k == "bicubic") {
        ks.kernel = Kernel::Bicubic;
        ks.support = 2.0;
        ks.kp1 = given(a.b) ? a.b : 0.0;
        ks.kp2 = given(a.c) ? a.c : 0.6;
    } else if (k == "lanczos") {
        ks.kernel = Kernel::Lanczos;
        const long taps = given(a.taps) ? a.taps : 3;
        if (taps < 1 || taps > 64)
            return fail("LGCR: lanczos taps must be in the range 1..64");
        ks.kp1 = double(taps);
        ks.support = ks.kp1;
    } else if (k == "spline16") {
        ks.kernel = Kernel::Spline16;
        ks.support = 2.0;
    } else if (k == "spline36") {
        ks.kernel = Kernel::Spline36;
        ks.support = 3.0;
    } else if (k == "jinc") {
        ks.kernel = Kernel::Jinc;
        ks.radial = true;
        const long taps = given(a.taps) ? a.taps : 3;
        if (taps < 1 || taps > 64)
            return fail("LGCR: jinc taps must be in the range 1..64");
        ks.kp1 = double(taps);
        ks.support = ks.kp1;
        const int n = static_cast<int>(ks.support * 1024) + 2;
        ks.lut.resize(n);
        for (int i = 0; i < n; ++i)
            ks.lut[i] = static_cast<float>(jincWindowed(double(i) / 1024.0, ks.support));
        ks.lutScale = 1024.0f;
    } else {
        return fail("LGCR: kernel must be \"bilinear\", \"bicubic\", \"lanczos\", \"spline16\", "
                    "\"spline36\" or \"jinc\"");
    }
    d.taps = 2 * static_cast<int>(std::ceil(ks.support));
    d.strength = given(a.strength) ? a.strength : 0.8;
    d.sigma = given(a.sigma) ? a.sigma : 0.01;
    d.sratio = given(a.sratio) ? a.sratio : 0.15;
    d.algo = given(a.algo) ? a.algo : 2;
    if (d.algo != 2 && d.algo != 4 && d.algo != 6)
        return fail("LGCR: algo must be 2 (guided), 4 (selector) or 6 (detail transfer)");
    d.sdb = given(a.sdb) ? a.sdb : 3.0;
    d.stretch = given(a.stretch) ? a.stretch : 1.0;
    d.gsigma = given(a.gsigma) ? a.gsigma : 2.5;
    d.rescue = given(a.rescue) ? a.rescue : 1.0;
    d.ridge = given(a.ridge) ? (a.ridge != 0) : true;
    d.cedge = given(a.cedge) ? (a.cedge != 0) : false;
    d.ms = given(a.ms) ? a.ms : 1.0;
    d.qgate = given(a.qgate) ? a.qgate : 1.0;
    d.arMargin = given(a.ar) ? a.ar : 0.0;
    d.reg = given(a.reg) ? a.reg : 0.005;
    if (a.loc) {
        const std::string l = a.loc;
        if (l == "left") d.shiftX = -0.5;
        else if (l == "center") d.shiftX = 0.0;
        else return fail("LGCR: loc must be \"left\" or \"center\"");
        d.locSet = true;
    } else {
        d.shiftX = -0.5;
    }
    d.sparse = given(a.sparse) ? (a.sparse != 0) : true;
    d.bm = given(a.bm) ? (a.bm != 0) : false;
    d.bp = given(a.bp) ? a.bp : 0.0;
    if (fmt->subsampling_w == 0)
        d.shiftX = 0.0;
    if (fmt->subsampling_h == 0)
        d.shiftY = 0.0;
    if (d.strength < 0.0 || d.strength > 1.0 || d.sigma <= 0.0 || d.sratio <= 0.0 ||
        d.sdb <= 0.0 || d.stretch < 0.0 || d.gsigma <= 0.0 || d.reg <= 0.0 ||
        d.bp < 0.0 || d.bp > 1.0 || d.ms < 0.0 || d.ms > 1.0 ||
        d.qgate < 0.0 || d.qgate > 1.0 || d.rescue < 0.0 || d.rescue > 1.0)
        return fail("LGCR: invalid parameter range (need 0<=strength/rescue<=1, 0<=bp/ms/qgate<=1, "
                    "sigma/sratio/sdb/gsigma/reg>0, stretch>=0)");

    // device-path limits (no reference counterpart): work lists pack output
    // coordinates into 16 bits, mask rows span at most kDilMaxWords words
    if (fmt->width > 65535 || fmt->height > 65535 || d.outW > 65535 || d.outH > 65535)
        return fail("LGCR: frame dimensions above 65535 are not supported on the device path");
    if (int(std::ceil(ks.support * 2.0)) + 8 >= 32 * kDilPadWords)
        return fail("LGCR: kernel support too large for the trust-mask dilation");

    f->sw = fmt->width;
    f->sh = fmt->height;
    f->cw = (fmt->width + (1 << fmt->subsampling_w) - 1) >> fmt->subsampling_w;
    f->ch = (fmt->height + (1 << fmt->subsampling_h) - 1) >> fmt->subsampling_h;
    if (!ks.lut.empty()) {
        cudaError_t e = cudaMalloc(&f->dLut, ks.lut.size() * sizeof(float));
        if (e != cudaSuccess) { err = std::string("LGCR: ") + cudaGetErrorString(e); return LGCR_E_NOMEM; }
        e = cudaMemcpy(f->dLut, ks.lut.data(), ks.lut.size() * sizeof(float), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { err = std::string("LGCR: ") + cudaGetErrorString(e); return LGCR_E_CUDA; }
    }
    *out = f.release();
    return LGCR_OK;
}

// applyFrameChromaSiting, src/plugin.cpp:157-175
FilterParams Filter::sited(int cl) const {
    FilterParams q = p;
    if (fmt.subsampling_w == 0) q.shiftX = 0.0;
    if (fmt.subsampling_h == 0) q.shiftY = 0.0;
    if (q.locSet || cl < 0)
        return q;
    if (fmt.subsampling_w > 0)
        q.shiftX = (cl == 0 || cl == 2 || cl == 4) ? -0.5 : 0.0;
    if (fmt.subsampling_h > 0)
        q.shiftY = (cl == 2 || cl == 3) ? -0.5 : (cl == 4 || cl == 5) ? 0.5 : 0.0;
    return q;
}

bool Filter::needsBackProjection(const FilterParams &q) const {
    return q.bp > 0.0 && q.outW == sw && q.outH == sh && cw * 2 == sw && ch * 2 == sh;
}

bool Filter::directOutput(const FilterParams &q) const {
    if (q.bm || needsBackProjection(q))
        return false;
    return q.strength == 0.0 || q.algo == 2 || (q.algo == 4 && !isFloat());
}

// ---------------------------------------------------------------------------
// resident tables
// ---------------------------------------------------------------------------
namespace {

// Host image of a table arena: arrays are appended with their offsets.
struct Packer {
    std::vector<uint8_t> bytes;
    template <class T> size_t add(const std::vector<T> &v) {
        const size_t off = (bytes.size() + 255) & ~size_t(255);
        bytes.resize(off + v.size() * sizeof(T));
        if (!v.empty())
            std::memcpy(bytes.data() + off, v.data(), v.size() * sizeof(T));
        return off;
    }
};

struct AxisOffsets { size_t start, w, wd, am, wsum, wabs, pos, lpos, cbI0, cbF, lbI0, lbF, kmx, kss, amBits; int n, sup; };

AxisOffsets packAxis(Packer &pk, const ChromaAxis &a) {
    AxisOffsets o;
    o.n = a.n; o.sup = a.sup;
    const std::vector<double> wd(a.w.begin(), a.w.end());
    o.start = pk.add(a.start); o.w = pk.add(a.w); o.wd = pk.add(wd); o.am = pk.add(a.am);
    o.wsum = pk.add(a.weightSum); o.wabs = pk.add(a.absoluteWeightSum);
    o.pos = pk.add(a.pos); o.lpos = pk.add(a.lpos);
    o.cbI0 = pk.add(a.chromaBilin.i0); o.cbF = pk.add(a.chromaBilin.f);
    o.lbI0 = pk.add(a.lumaBilin.i0); o.lbF = pk.add(a.lumaBilin.f);
    std::vector<float> kmx, kss;
    rescueFactors(a, kmx, kss);
    o.kmx = pk.add(kmx); o.kss = pk.add(kss);
    // tap activity of each index as one word (the same bits as the bytes)
    std::vector<uint32_t> bits(a.sup <= 32 ? size_t(a.n) : 0, 0u);
    for (size_t i = 0; i < bits.size(); ++i)
        for (int j = 0; j < a.sup; ++j)
            if (a.am[i * a.sup + j])
                bits[i] |= 1u << j;
    o.amBits = pk.add(bits);
    return o;
}

AxisView axisView(const DeviceArena &ar, const AxisOffsets &o) {
    AxisView v;
    v.n = o.n; v.sup = o.sup;
    v.start = (const int *)ar.at(o.start); v.w = (const float *)ar.at(o.w);
    v.wd = (const double *)ar.at(o.wd);
    v.am = (const uint8_t *)ar.at(o.am); v.wsum = (const float *)ar.at(o.wsum);
    v.wabs = (const float *)ar.at(o.wabs); v.pos = (const float *)ar.at(o.pos);
    v.lpos = (const float *)ar.at(o.lpos); v.cbI0 = (const int *)ar.at(o.cbI0);
    v.cbF = (const float *)ar.at(o.cbF); v.lbI0 = (const int *)ar.at(o.lbI0);
    v.lbF = (const float *)ar.at(o.lbF);
    v.kmx = (const float *)ar.at(o.kmx); v.kss = (const float *)ar.at(o.kss);
    v.amBits = o.sup <= 32 ? (const uint32_t *)ar.at(o.amBits) : nullptr;
    return v;
}

struct WeightOffsets { size_t start, w; int n, sup; };
WeightOffsets packWeights(Packer &pk, const WeightTable &t) {
    return { pk.add(t.start), pk.add(t.w), t.n, t.sup };
}
WeightView weightView(const DeviceArena &ar, const WeightOffsets &o) {
    return { o.n, o.sup, (const int *)ar.at(o.start), (const float *)ar.at(o.w) };
}

struct RadialOffsets { size_t xPhase, yPhase, weights, kappa; int valid, supX, supY, phasesX; };
RadialOffsets packRadial(Packer &pk, const RadialTable &t) {
    RadialOffsets o{};
    o.valid = t.valid;
    o.supX = t.supportX; o.supY = t.supportY; o.phasesX = t.phaseCountX;
    if (t.valid) {
        o.xPhase = pk.add(t.xPhase); o.yPhase = pk.add(t.yPhase); o.weights = pk.add(t.weights);
        o.kappa = pk.add(t.kappa);
    }
    return o;
}
RadialView radialView(const DeviceArena &ar, const RadialOffsets &o) {
    RadialView v{};
    v.valid = o.valid;
    v.supX = o.supX; v.supY = o.supY; v.phasesX = o.phasesX;
    if (o.valid) {
        v.xPhase = (const uint16_t *)ar.at(o.xPhase);
        v.yPhase = (const uint16_t *)ar.at(o.yPhase);
        v.weights = (const float *)ar.at(o.weights);
        v.kappa = (const float *)ar.at(o.kappa);
    }
    return v;
}

} // namespace

void setAxisGeometry(DeviceTables &t, const ChromaAxis &ax, const ChromaAxis &ay, int outH,
                     int ch) {
    t.axSup = ax.sup;
    t.aySup = ay.sup;
    // k_plain blocks: tall when every block's chroma rows fit in shared memory
    auto plainRowsRead = [&](int rows) {
        int most = 0;
        for (int oy0 = 0; oy0 < outH; oy0 += rows) {
            const int oyLast = std::min(oy0 + rows, outH) - 1;
            const int lo = std::clamp(ay.start[oy0], 0, ch - 1);
            const int hi = std::clamp(ay.start[oyLast] + ay.sup - 1, 0, ch - 1);
            most = std::max(most, hi - lo + 1);
        }
        return most;
    };
    t.plainRows = kPlainRowsShort;
    t.plainMaxRows = plainRowsRead(kPlainRowsShort);
    for (int rows = kPlainRows; rows > kPlainRowsShort; rows -= 8) {
        const int most = plainRowsRead(rows);
        if (most <= kPlainStagedRows) {
            t.plainRows = rows;
            t.plainMaxRows = most;
            break;
        }
    }
}

const DeviceTables *Filter::tablesFor(double shiftX, double shiftY) {
    std::lock_guard<std::mutex> lock(mu);
    for (auto &t : tables)
        if (t->shiftX == shiftX && t->shiftY == shiftY)
            return t.get();
    auto t = std::make_unique<DeviceTables>();
    t->shiftX = shiftX;
    t->shiftY = shiftY;
    const double rw = double(sw) / cw, rh = double(sh) / ch;
    const ChromaAxis ax = buildChromaAxis(sw, p.outW, rw, shiftX, p.k);
    const ChromaAxis ay = buildChromaAxis(sh, p.outH, rh, shiftY, p.k);
    Packer pk;
    const AxisOffsets oax = packAxis(pk, ax), oay = packAxis(pk, ay);
    RadialOffsets orad{};
    if (p.k.radial)
        orad = packRadial(pk, buildRadialTable(p.k, ax, ay, cw, ch));
    const bool sameSize = p.outW == sw && p.outH == sh;
    WeightOffsets olh{}, olv{};
    if (!sameSize && !p.k.radial) {
        olh = packWeights(pk, buildWeights(sw, p.outW, p.k, 0.0));
        olv = packWeights(pk, buildWeights(sh, p.outH, p.k, 0.0));
    }
    // algo 6: degradation candidates, source-grid plain axes, Nyquist levels
    const bool algo6 = p.algo == 6 && p.strength > 0.0;
    WeightOffsets oy1h{}, oy1v{}, oy2h{}, oy2v{};
    AxisOffsets osax{}, osay{};
    RadialOffsets osrad{};
    if (algo6) {
        KernelSpec bil;
        bil.kernel = Kernel::Bilinear; bil.kp1 = bil.kp2 = 0.0; bil.support = 1.0;
        KernelSpec bic;
        bic.kernel = Kernel::Bicubic; bic.kp1 = 0.0; bic.kp2 = 0.6; bic.support = 2.0;
        const WeightTable y1h = buildWeights(sw, cw, bil, shiftX), y1v = buildWeights(sh, ch, bil, shiftY);
        const WeightTable y2h = buildWeights(sw, cw, bic, shiftX), y2v = buildWeights(sh, ch, bic, shiftY);
        oy1h = packWeights(pk, y1h);
        oy1v = packWeights(pk, y1v);
        oy2h = packWeights(pk, y2h);
        oy2v = packWeights(pk, y2v);
        t->ycMaxSup = std::max(std::max(y1h.sup, y1v.sup), std::max(y2h.sup, y2v.sup));
        for (int c0 = 0; c0 < ch; c0 += kYcTile) {
            const int c1 = std::min(c0 + kYcTile, ch) - 1;
            for (const WeightTable *v : {&y1v, &y2v}) {
                const int lo = std::clamp(v->start[c0], 0, sh - 1);
                const int hi = std::clamp(v->start[c1] + v->sup - 1, 0, sh - 1);
                t->ycMaxRows = std::max(t->ycMaxRows, hi - lo + 1);
            }
        }
        const ChromaAxis sax = buildChromaAxis(sw, sw, rw, shiftX, p.k);
        const ChromaAxis say = buildChromaAxis(sh, sh, rh, shiftY, p.k);
        osax = packAxis(pk, sax);
        osay = packAxis(pk, say);
        t->sAxSup = sax.sup;
        t->sAySup = say.sup;
        auto detailRowsRead = [&](int rows) {
            int most = 0;
            for (int y0 = 0; y0 < sh; y0 += rows) {
                const int r0 = std::clamp(y0 - 1, 0, sh - 1), r1 = std::clamp(y0 + rows, 0, sh - 1);
                const int lo = std::clamp(say.start[r0], 0, ch - 1);
                const int hi = std::clamp(say.start[r1] + say.sup - 1, 0, ch - 1);
                most = std::max(most, hi - lo + 1);
            }
            return most;
        };
        t->detailRows = kDetailRowsTall;
        t->detailMaxRows = detailRowsRead(kDetailRowsTall);
        if (t->detailMaxRows > kDetailStagedRows) {
            t->detailRows = kDetailTile;
            t->detailMaxRows = detailRowsRead(kDetailTile);
        }
        if (p.k.radial)
            osrad = packRadial(pk, buildRadialTable(p.k, sax, say, cw, ch));
    }
    // algo 4: point-sampled luma positions (pointSampledLuma, algos.cpp:300-315)
    const bool algo4 = p.algo == 4 && p.strength > 0.0;
    size_t olsX = 0, olsXf = 0, olsY = 0, olsYf = 0;
    if (algo4) {
        std::vector<float> xPos(cw), yPos(ch);
        for (int x = 0; x < cw; ++x)
            xPos[x] = float((x + 0.5) * rw - 0.5 + shiftX);
        for (int y = 0; y < ch; ++y)
            yPos[y] = float((y + 0.5) * rh - 0.5 + shiftY);
        const BilinAxis bx = buildBilinAxis(xPos, sw), by = buildBilinAxis(yPos, sh);
        olsX = pk.add(bx.i0); olsXf = pk.add(bx.f);
        olsY = pk.add(by.i0); olsYf = pk.add(by.f);
    }
    // bm: 8-px anchor grid plus the last full patch (blockStarts, bm.cpp:214-224)
    auto blockStarts = [](int extent) {
        std::vector<int> starts;
        if (extent < 8)
            return starts;
        const int last = extent - 8;
        for (int pos = 0; pos <= last; pos += 8)
            starts.push_back(pos);
        if (starts.empty() || starts.back() != last)
            starts.push_back(last);
        return starts;
    };
    const std::vector<int> bmX = p.bm ? blockStarts(p.outW) : std::vector<int>{};
    const std::vector<int> bmY = p.bm ? blockStarts(p.outH) : std::vector<int>{};
    const size_t obmX = pk.add(bmX), obmY = pk.add(bmY);
    std::vector<int> xb, xe, yb, ye;
    lcExtents(sw, cw, rw, shiftX, xb, xe);
    lcExtents(sh, ch, rh, shiftY, yb, ye);
    const size_t oxb = pk.add(xb), oxe = pk.add(xe), oyb = pk.add(yb), oye = pk.add(ye);

    t->arena.reserve(pk.bytes.size());
    if (!t->arena.commit())
        return nullptr;
    if (cudaMemcpy(t->arena.at(0), pk.bytes.data(), pk.bytes.size(), cudaMemcpyHostToDevice) !=
        cudaSuccess)
        return nullptr;
    t->ax = axisView(t->arena, oax);
    t->ay = axisView(t->arena, oay);
    setAxisGeometry(*t, ax, ay, p.outH, ch);
    if (p.k.radial)
        t->rad = radialView(t->arena, orad);
    if (!sameSize && !p.k.radial) {
        t->lumaH = weightView(t->arena, olh);
        t->lumaV = weightView(t->arena, olv);
    }
    if (algo6) {
        t->ycH1 = weightView(t->arena, oy1h);
        t->ycV1 = weightView(t->arena, oy1v);
        t->ycH2 = weightView(t->arena, oy2h);
        t->ycV2 = weightView(t->arena, oy2v);
        t->sax = axisView(t->arena, osax);
        t->say = axisView(t->arena, osay);
        if (p.k.radial)
            t->srad = radialView(t->arena, osrad);
        auto levels = [](double ratio) {
            int n = 0;
            while (ratio > 1.5 && n < 4) { ratio *= 0.5; ++n; }
            return n;
        };
        t->nyqX = levels(rw);
        t->nyqY = levels(rh);
    }
    if (algo4) {
        t->lsX = (const int *)t->arena.at(olsX);
        t->lsXf = (const float *)t->arena.at(olsXf);
        t->lsY = (const int *)t->arena.at(olsY);
        t->lsYf = (const float *)t->arena.at(olsYf);
    }
    if (p.bm && !bmX.empty() && !bmY.empty()) {
        t->bmStartsX = (const int *)t->arena.at(obmX);
        t->bmStartsY = (const int *)t->arena.at(obmY);
        t->bmAnchorsX = int(bmX.size());
        t->bmAnchorsY = int(bmY.size());
    }
    t->lcXb = (const int *)t->arena.at(oxb);
    t->lcXe = (const int *)t->arena.at(oxe);
    t->lcYb = (const int *)t->arena.at(oyb);
    t->lcYe = (const int *)t->arena.at(oye);
    tables.push_back(std::move(t));
    return tables.back().get();
}

// ---------------------------------------------------------------------------
// workspaces
// ---------------------------------------------------------------------------
std::unique_ptr<Workspace> Filter::makeWorkspace(bool hostStaging) {
    auto ws = std::make_unique<Workspace>();
    ws->owner = this;
    DeviceArena &ar = ws->arena;
    const size_t L = size_t(sw) * sh, C = size_t(cw) * ch, O = size_t(p.outW) * p.outH;
    const bool guided = p.strength > 0.0;
    const bool sameSize = p.outW == sw && p.outH == sh;
    const int bps = bytesPerSample();
    struct Slot { size_t off = 0; bool on = false; };
    auto take = [&](size_t bytes, bool on = true) { Slot s; s.on = on; if (on) s.off = ar.reserve(bytes); return s; };
    Slot sJob = take(sizeof(FrameJob));
    Slot sY = take(L * 4), sU = take(C * 4), sV = take(C * 4);
    Slot sJxx = take(L * 4, guided), sJxy = take(L * 4, guided), sJyy = take(L * 4, guided);
    Slot sLc = take(C * 4, guided), sMs = take(C * 4, guided && p.ms > 0.0);
    const bool sparse = guided && p.sparse;
    const size_t maskBytes = size_t((sw + 31) / 32) * 4 * sh;
    Slot sSeed = take(L, sparse), sMtmp = take(maskBytes, sparse), sMask = take(maskBytes, sparse);
    Slot sCmask = take(C, sparse);
    Slot sOU = take(O * 4), sOV = take(O * 4);
    Slot sLumaTmp = take(size_t(p.outW) * sh * 4, !sameSize && !p.k.radial);  // luma / detail resize
    Slot sCnt = take(kCntCount * sizeof(unsigned long long));
    const bool listed = guided && (p.algo == 2 || p.algo == 4);
    Slot sUvd = take(C * 16), sHTab = take(size_t(p.outW) * ch * 32, !p.k.radial);
    Slot sWExt = take(O * 24, listed && !p.k.radial && p.k.kernel != Kernel::Bilinear);
    Slot sList = take(O * 4, listed || (guided && p.algo == 6 && p.sparse));
    Slot sCList = take(C * 4, guided && p.algo == 6 && p.sparse);
    const bool algo6 = guided && p.algo == 6, algo4 = guided && p.algo == 4;
    Slot sAff = take(9 * C * 4, algo6), sYc1 = take(C * 4, algo6), sYc2 = take(C * 4, algo6);
    Slot sDt1 = take(L * 4, algo6), sDt2 = take(L * 4, algo6);
    Slot sDet = take(O * 4, algo6 && !sameSize);
    Slot sDTab = take(size_t(sw) * ch * 16, algo6 && !p.k.radial && p.k.kernel != Kernel::Bilinear);
    Slot sLumaTmp2 = take(size_t(p.outW) * sh * 4, algo6 && !sameSize && !p.k.radial && false);
    Slot sLgf = take(6 * C * 4, algo4);
    const bool sel = algo4 && isFloat();
    Slot sW2 = take(O * 4, sel), sW3 = take(O * 4, sel), sGU = take(O * 4, sel), sGV = take(O * 4, sel);
    Slot sRoi = take(C, sel);
    const size_t anchors = p.bm ? size_t((p.outW + 15) / 8) * ((p.outH + 15) / 8) : 0;
    Slot sBmG = take(anchors * 9 * sizeof(int), p.bm), sBmP = take(anchors * 520 * 4, p.bm);
    Slot sIn[3], sOut[3];
    for (int i = 0; i < 3; ++i) {
        const size_t n = i == 0 ? L : C;
        sIn[i] = take(n * bps, hostStaging);
        sOut[i] = take(O * bps, hostStaging);
    }
    if (!ar.commit())
        return nullptr;
    // LGCR_POISON_WORKSPACE=1: fill new workspaces with 0xFF bytes (NaN
    // floats, -1 integers), so a stage that reads scratch no stage wrote
    // shows in the output instead of depending on earlier frames
    if (const char *e = std::getenv("LGCR_POISON_WORKSPACE"); e && e[0] == '1')
        if (cudaMemset(ar.at(0), 0xFF, ar.size()) != cudaSuccess)
            return nullptr;
    auto F = [&](const Slot &s) { return s.on ? (float *)ar.at(s.off) : nullptr; };
    auto B = [&](const Slot &s) { return s.on ? (uint8_t *)ar.at(s.off) : nullptr; };
    ws->dJob = (FrameJob *)ar.at(sJob.off);
    ws->Yw = F(sY); ws->Uw = F(sU); ws->Vw = F(sV);
    ws->jxx = F(sJxx); ws->jxy = F(sJxy); ws->jyy = F(sJyy);
    ws->lc = F(sLc); ws->ms = F(sMs);
    ws->seed = B(sSeed); ws->mtmp = B(sMtmp); ws->mask = B(sMask); ws->cmask = B(sCmask);
    ws->oU = F(sOU); ws->oV = F(sOV); ws->lumaTmp = F(sLumaTmp);
    ws->counters = (unsigned long long *)ar.at(sCnt.off);
    ws->uvd = sUvd.on ? (double *)ar.at(sUvd.off) : nullptr;
    ws->hTab = F(sHTab);
    ws->wExt = F(sWExt);
    ws->actList = sList.on ? (uint32_t *)ar.at(sList.off) : nullptr;
    ws->chromaList = sCList.on ? (uint32_t *)ar.at(sCList.off) : nullptr;
    ws->aff = F(sAff); ws->yc1 = F(sYc1); ws->yc2 = F(sYc2);
    ws->detailTmp = F(sDt1); ws->detailTmp2 = F(sDt2); ws->detail = F(sDet); ws->dTab = F(sDTab);
    (void)sLumaTmp2;
    ws->lgf = F(sLgf);
    ws->selW2 = F(sW2); ws->selW3 = F(sW3); ws->gU = F(sGU); ws->gV = F(sGV);
    ws->roi = B(sRoi);
    ws->bmGroups = sBmG.on ? (int *)ar.at(sBmG.off) : nullptr;
    ws->bmPatch = F(sBmP);
    for (int i = 0; i < 3; ++i) {
        const int w = i == 0 ? sw : cw;
        ws->stageIn[i] = sIn[i].on ? ar.at(sIn[i].off) : nullptr;
        ws->stageInPitch[i] = size_t(w) * bps;
        ws->stageOut[i] = sOut[i].on ? ar.at(sOut[i].off) : nullptr;
        ws->stageOutPitch[i] = size_t(p.outW) * bps;
    }
    if (cudaEventCreateWithFlags(&ws->done, cudaEventDisableTiming) != cudaSuccess)
        return nullptr;
    if (cudaHostAlloc((void **)&ws->hJob, sizeof(FrameJob), cudaHostAllocDefault) != cudaSuccess)
        return nullptr;
    return ws;
}

// Prefer an idle workspace whose last frame has finished on the device; grow
// the pool (up to a few per filter) rather than wait for one in flight.
Workspace *Filter::acquire(bool hostStaging) {
    constexpr int kMaxWorkspaces = 4;
    auto &pool = hostStaging ? idle : idleBatch;
    auto &count = hostStaging ? live : liveBatch;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (size_t i = 0; i < pool.size(); ++i) {
            Workspace *ws = pool[i].get();
            if (!ws->used || cudaEventQuery(ws->done) == cudaSuccess) {
                pool[i].release();
                pool.erase(pool.begin() + i);
                return ws;
            }
        }
        if (count.load() >= kMaxWorkspaces && !pool.empty()) {
            Workspace *ws = pool.front().release();
            pool.erase(pool.begin());
            return ws;   // caller orders its work after the event
        }
    }
    auto ws = makeWorkspace(hostStaging);
    if (ws) {
        ws->hostStaging = hostStaging;
        count.fetch_add(1);
    }
    return ws.release();
}

void Filter::release(Workspace *ws) {
    if (!ws)
        return;
    std::lock_guard<std::mutex> lock(mu);
    (ws->hostStaging ? idle : idleBatch).emplace_back(ws);
}

// ---------------------------------------------------------------------------
// FrameJob
// ---------------------------------------------------------------------------
static int sampleKind(const lgcr_format &f) {
    if (f.sample_type == LGCR_ST_FLOAT) return kF32;
    return f.bits_per_sample > 8 ? kU16 : kU8;
}

void buildJob(const FrameTask &t, FrameJob &J) {
    std::memset(&J, 0, sizeof(J));
    const Filter &F = *t.filter;
    const FilterParams &p = t.p;
    const DeviceTables &T = *t.tables;
    Workspace &ws = *t.ws;
    J.sw = F.sw; J.sh = F.sh; J.cw = F.cw; J.ch = F.ch; J.W = p.outW; J.H = p.outH;
    J.rw = double(F.sw) / F.cw;
    J.rh = double(F.sh) / F.ch;
    J.rwF = float(J.rw);
    J.rhF = float(J.rh);
    J.sameSize = (J.W == J.sw && J.H == J.sh);
    J.inKind = J.outKind = sampleKind(F.fmt);
    J.bits = F.fmt.bits_per_sample;
    const bool isFloat = F.isFloat();
    J.yScale = isFloat ? 1.0 : 1.0 / double((1 << J.bits) - 1);
    J.cOffset = isFloat ? 0.0 : -0.5;
    const double outScale = isFloat ? 1.0 : double((1 << J.bits) - 1);
    J.qScale = float(outScale);
    J.qOffC = float(isFloat ? 0.0 : 0.5 * outScale);
    J.maxCode = isFloat ? 0 : (1 << J.bits) - 1;
    for (int i = 0; i < 3; ++i) {
        J.in[i] = t.in[i].data;
        J.inPitch[i] = t.in[i].stride;
        J.out[i] = t.out[i].data;
        J.outPitch[i] = t.out[i].stride;
    }
    J.writeLuma = t.out[0].data != nullptr;

    J.algo = p.algo;
    J.kernel = int(p.k.kernel);
    J.radial = p.k.radial;
    J.guided = p.strength > 0.0;
    J.sparse = J.guided && p.sparse;
    J.ridge = p.ridge;
    J.cedge = p.cedge;
    J.bm = p.bm;
    J.useMs = J.guided && p.ms > 0.0;
    J.clampHull = p.arMargin >= 0.0;
    J.trustOn = J.sparse;
    const double trustThreshold = p.algo == 4 ? 0.25 * p.sigma : p.sigma;
    J.trustThr = float(trustThreshold * trustThreshold);
    J.dil = int(std::ceil(p.k.support * std::max(J.rw, J.rh))) + 8;
    J.directOutput = F.directOutput(p);
    J.needBackProject = F.needsBackProjection(p);
    J.strength = p.algo == 4 ? 1.0f : float(p.strength);
    J.strength4 = float(p.strength);
    J.support = p.k.support;
    J.sigma = float(p.sigma);
    J.sratio = float(p.sratio);
    J.sdb = float(p.sdb);
    J.stretch = float(p.stretch);
    J.invGsigma2 = 1.0f / float(p.gsigma * p.gsigma);
    J.rescue = float(p.rescue);
    J.msStrength = float(p.ms);
    J.qgate = float(p.qgate);
    J.margin = float(std::max(0.0, p.arMargin));
    J.spOut = float(std::max(J.rw, J.rh));
    J.bpGain = float(p.bp);
    J.invWxC = float(std::min(1.0, double(J.W) / F.cw));
    J.invWyC = float(std::min(1.0, double(J.H) / F.ch));
    J.lut = F.dLut;
    J.lutN = int(p.k.lut.size());
    J.lutScale = p.k.lutScale;
    J.lgfEps = p.reg * p.reg;

    J.ax = T.ax; J.ay = T.ay; J.rad = T.rad;
    J.lumaH = T.lumaH; J.lumaV = T.lumaV;
    J.lcXb = T.lcXb; J.lcXe = T.lcXe; J.lcYb = T.lcYb; J.lcYe = T.lcYe;

    // float input planes that are already packed are read in place
    const bool packedY = isFloat && t.in[0].stride == (ptrdiff_t)F.sw * 4;
    const bool packedU = isFloat && t.in[1].stride == (ptrdiff_t)F.cw * 4;
    const bool packedV = isFloat && t.in[2].stride == (ptrdiff_t)F.cw * 4;
    J.Yw = packedY ? nullptr : ws.Yw;
    J.Uw = packedU ? nullptr : ws.Uw;
    J.Vw = packedV ? nullptr : ws.Vw;
    J.Y = packedY ? (const float *)t.in[0].data : ws.Yw;
    J.U = packedU ? (const float *)t.in[1].data : ws.Uw;
    J.V = packedV ? (const float *)t.in[2].data : ws.Vw;
    J.jxx = ws.jxx; J.jxy = ws.jxy; J.jyy = ws.jyy;
    J.lc = ws.lc; J.ms = ws.ms;
    J.seed = ws.seed; J.cmask = ws.cmask;
    J.mtmp = reinterpret_cast<uint32_t *>(ws.mtmp);
    J.mask = reinterpret_cast<uint32_t *>(ws.mask);
    J.maskWords = (F.sw + 31) / 32;
    J.oU = ws.oU; J.oV = ws.oV; J.lumaTmp = ws.lumaTmp;
    J.counters = ws.counters;
    J.uvd = ws.uvd;
    J.hTab = ws.hTab;
    J.actList = ws.actList;
    J.listed = J.guided && (p.algo == 2 || p.algo == 4);
    J.xferListed = (J.guided && p.algo == 6 && J.sparse && ws.actList) ? 1 : 0;
    // upscaling frames (output >= 2x the source luma) list their pixels in row
    // groups: every chroma sample feeds many output rows there, and a guided
    // block's pixels then share their windows in L1 (1080p -> 4K jinc guided
    // pass 9-11 % faster); same-size sparse frames keep the raster order,
    // whose warps store one row segment each (row groups cost them 1 %)
    J.listGroup = ((long long)J.W * J.H >= 2LL * J.sw * J.sh) ? kListRowGroup : 1;
    J.chromaList = (J.guided && p.algo == 6 && J.sparse) ? ws.chromaList : nullptr;
    {
        // guided bump denominator 1 + dp^2/g^2 + dt^2/(g*aniso)^2 with aniso >= 1:
        // |dp|, |dt| <= (tap distance in chroma samples) * ratio * |n| summed
        // over both axes; bound it with margin well below 2^64
        const double d = double(std::max(T.axSup, T.aySup) + 2) * std::max(J.rw, J.rh) * 2.0 * 1.01;
        const double bound = 1.0 + 2.0 * d * d * double(J.invGsigma2);
        J.bumpRcpSafe = bound < 1.0e18 ? 1 : 0;
    }
    J.plainFused = (J.hTab && !J.radial && T.plainMaxRows <= kPlainStagedRows) ? 1 : 0;
    J.plainRows = J.plainFused ? T.plainRows : kPlainRowsShort;
    J.wHull = nullptr;
    J.wLum = nullptr;
    if (ws.wExt && J.listed && J.plainFused && J.kernel != 0 && T.aySup <= 8) {
        // k_plain folds the guided windows' extrema for the listed pixels from
        // its staged rows; the horizontal table is then only needed for the
        // integer algo 4 plain base the guided pass recomputes
        J.wHull = reinterpret_cast<float4 *>(ws.wExt);
        J.wLum = reinterpret_cast<float2 *>(ws.wExt + size_t(J.W) * J.H * 4);
        if (!(p.algo == 4 && J.outKind != kF32))
            J.hTab = nullptr;
    }
    {
        // every tap index in range: starts lie in [0, srcChromaN - sup] and the
        // integer-ratio chroma count equals the plane size
        const int nx = (F.sw + int(J.rw) - 1) / int(J.rw);
        const int ny = (F.sh + int(J.rh) - 1) / int(J.rh);
        J.noClampX = (nx == F.cw && F.cw >= T.axSup) ? 1 : 0;
        J.noClampY = (ny == F.ch && F.ch >= T.aySup) ? 1 : 0;
    }
    // algo 6
    J.aff = ws.aff; J.yc1 = ws.yc1; J.yc2 = ws.yc2;
    J.detailTmp = ws.detailTmp; J.detailTmp2 = ws.detailTmp2; J.dTab = ws.dTab;
    J.ycH1 = T.ycH1; J.ycV1 = T.ycV1; J.ycH2 = T.ycH2; J.ycV2 = T.ycV2;
    J.sax = T.sax; J.say = T.say; J.srad = T.srad;
    J.nyqX = T.nyqX; J.nyqY = T.nyqY;
    J.sinvWxC = float(std::min(1.0, double(F.sw) / F.cw));
    J.sinvWyC = float(std::min(1.0, double(F.sh) / F.ch));
    J.epsSig = (0.25 * p.sigma) * (0.25 * p.sigma);
    if (p.algo == 6 && J.guided) {
        const float *last = ((J.nyqX + J.nyqY) & 1) ? ws.detailTmp2 : ws.detailTmp;
        J.detailSrc = last;
        J.detail = J.sameSize ? const_cast<float *>(last) : ws.detail;
        const int nx = (F.sw + int(J.rw) - 1) / int(J.rw);
        const int ny = (F.sh + int(J.rh) - 1) / int(J.rh);
        J.sNoClampX = (nx == F.cw && F.cw >= T.sAxSup) ? 1 : 0;
        J.sNoClampY = (ny == F.ch && F.ch >= T.sAySup) ? 1 : 0;
        J.ycTiled = (T.ycMaxSup <= 8 && T.ycMaxRows <= kYcRows) ? 1 : 0;
        J.detailRows = T.detailRows;
        J.detailFused = (J.dTab && !J.radial && J.kernel != 0 && T.sAxSup <= 8 && T.sAySup <= 8 &&
                         T.detailMaxRows <= kDetailStagedRows && J.nyqX <= 1 && J.nyqY <= 1) ? 1 : 0;
        // The detail transfer reads the map only at active pixels (sparse mask,
        // same-size output) and bilinearly at +-s along the edge tangent, with
        // s = 1 + stretch * coherence and coherence <= 1 (the smoothed tensor is
        // positive semi-definite; 0.1 % margin for rounding): samples more than
        // floor(1 + stretch) + 2 away from every active pixel are never read.
        J.detailReach = (J.sparse && J.sameSize)
            ? int(std::floor(1.0 + double(p.stretch) * 1.001)) + 2 : 0;
    }
    // algo 4
    J.lgf = ws.lgf;
    J.selW2 = ws.selW2; J.selW3 = ws.selW3; J.gU = ws.gU; J.gV = ws.gV;
    J.roi = ws.roi;
    J.lgfRoiOnly = (p.algo == 4 && isFloat) ? 1 : 0;
    J.lsX = T.lsX; J.lsXf = T.lsXf; J.lsY = T.lsY; J.lsYf = T.lsYf;
    // bm
    J.bmGroups = ws.bmGroups; J.bmPatch = ws.bmPatch;
    J.bmStartsX = T.bmStartsX; J.bmStartsY = T.bmStartsY;
    J.bmAnchorsX = T.bmAnchorsX; J.bmAnchorsY = T.bmAnchorsY;
    J.bmSigma = float(p.sigma);
    if (!T.bmStartsX)
        J.bm = 0;                                 // frame smaller than one patch
    // algo 6 with nothing after the detail transfer: the plain stage stores
    // the pixels the transfer leaves alone, the transfer stores the others
    J.finalInTransfer = (p.algo == 6 && J.guided && !J.bm && !J.needBackProject) ? 1 : 0;
    // float algo 4 with nothing after the blend: the blend stores every pixel
    J.blendStores = (J.guided && J.lgfRoiOnly && !J.bm && !J.needBackProject && !J.directOutput)
                        ? 1 : 0;
    // back-projection is the last stage when it runs, and each output pixel
    // lies in exactly one chroma sample's 2x2 block: it stores them
    J.bpStores = J.needBackProject ? 1 : 0;
}

// ---------------------------------------------------------------------------
// stage scheduler
// ---------------------------------------------------------------------------
enum StageId : int {
    S_CONVERT, S_LUMA_RADIAL, S_LUMA_H, S_LUMA_V, S_TENSOR, S_DIL_H, S_DIL_V,
    S_MARK, S_COUNT, S_GATE, S_LGF_DENSE, S_HPASS, S_PLAIN, S_GUIDED,
    S_YC, S_YC_TILED, S_AFFINE, S_AFFINE_LIST, S_DET_HPASS, S_DET_PLAIN, S_DET_MAP, S_NYQ0, S_NYQ1, S_NYQ2, S_NYQ3, S_NYQ4, S_NYQ5, S_NYQ6, S_NYQ7,
    S_DET_RH, S_DET_RV, S_DET_RR, S_DET_TRANSFER, S_DET_XFER_LIST,
    S_ROI, S_LGF_ROI, S_BLEND, S_BM_GROUP, S_BM_AGG, S_BP, S_STORE, S_N
};

int stageCount() { return S_N; }

// Stage names; the ones with a reference counterpart use the reference's
// stage vocabulary (stageName, src/pipeline.h:222-245).
const char *stageName(int s) {
    static const char *names[S_N] = {
        "input_conversion", "luma_resample_radial", "luma_resample_h", "luma_resample_v",
        "buildGuideMaps_tensor", "buildTrustMask_h", "buildTrustMask_v",
        "buildSparseWorkset", "buildSparseWorkset_count", "buildMutualGate", "buildLGF",
        "plainChroma_horizontal", "plainChroma", "reconstructChroma", "buildAffineMaps_candidates", "buildAffineMaps_candidates_tiled", "buildAffineMaps", "buildAffineMaps_listed", "buildDetail_horizontal", "buildDetail_plain", "buildDetailMap",
        "buildDetail_nyquist0", "buildDetail_nyquist1", "buildDetail_nyquist2", "buildDetail_nyquist3",
        "buildDetail_nyquist4", "buildDetail_nyquist5", "buildDetail_nyquist6", "buildDetail_nyquist7",
        "buildDetail_resize_h", "buildDetail_resize_v", "buildDetail_resize_radial", "detailTransfer",
        "detailTransfer_listed", "selector_roi", "buildLGF_roi", "selectorBlend", "collaborative_chroma_group",
        "collaborative_chroma", "backProject", "output_conversion",
    };
    return (s >= 0 && s < S_N) ? names[s] : "unknown";
}

static inline int cdiv(int a, int b) { return (a + b - 1) / b; }

// Launch shapes of the tunable per-pixel stages (process-wide; set by the
// autotuner). Other stages use fixed shapes tied to their shared tiles.
static std::mutex gShapeMu;
static int gShapeX[S_N], gShapeY[S_N];
static bool gShapeInit = false;

static void initShapes() {
    if (gShapeInit) return;
    for (int i = 0; i < S_N; ++i) { gShapeX[i] = 32; gShapeY[i] = 8; }
    gShapeInit = true;
}

bool stageTunable(int s) {
    return s == S_HPASS || s == S_AFFINE || s == S_DET_TRANSFER || s == S_DET_PLAIN ||
           s == S_LGF_DENSE || s == S_YC || s == S_BM_AGG;
}

void stageShape(int s, int &bx, int &by) {
    std::lock_guard<std::mutex> lock(gShapeMu);
    initShapes();
    bx = gShapeX[s]; by = gShapeY[s];
}

static std::atomic<int> gConfigVersion{0};

int processConfigVersion() { return gConfigVersion.load(); }

void setStageShape(int s, int bx, int by) {
    std::lock_guard<std::mutex> lock(gShapeMu);
    initShapes();
    gShapeX[s] = bx; gShapeY[s] = by;
    gConfigVersion.fetch_add(1);
}

// Variant of the persistent guided kernel (0: 2 blocks/SM, 1: 3 blocks/SM,
// 2: 2 blocks/SM with the warps' tap windows staged in shared memory).
// LGCR_GUIDED_VARIANT sets the initial choice.
static int gGuidedVariant = -1;

int guidedVariant() {
    std::lock_guard<std::mutex> lock(gShapeMu);
    if (gGuidedVariant < 0) {
        const char *e = std::getenv("LGCR_GUIDED_VARIANT");
        gGuidedVariant = (e && e[0] >= '0' && e[0] <= '2') ? e[0] - '0' : 0;
    }
    return gGuidedVariant;
}

void setGuidedVariant(int v) {
    std::lock_guard<std::mutex> lock(gShapeMu);
    gGuidedVariant = (v >= 0 && v <= 2) ? v : 0;
    gConfigVersion.fetch_add(1);
}

static_assert(S_N <= kMaxStages, "LaunchConfig holds every stage");

// One lock for the whole snapshot: every frame plan takes one, from as many
// host threads as call the library at once.
LaunchConfig processLaunchConfig() {
    LaunchConfig c;
    for (int s = 0; s < kMaxStages; ++s) {
        c.shapeX[s] = 32;
        c.shapeY[s] = 8;
    }
    std::lock_guard<std::mutex> lock(gShapeMu);
    initShapes();
    for (int s = 0; s < S_N; ++s) {
        c.shapeX[s] = gShapeX[s];
        c.shapeY[s] = gShapeY[s];
    }
    if (gGuidedVariant < 0) {
        const char *e = std::getenv("LGCR_GUIDED_VARIANT");
        gGuidedVariant = (e && e[0] >= '0' && e[0] <= '2') ? e[0] - '0' : 0;
    }
    c.guidedVariant = gGuidedVariant;
    return c;
}

static int stageTilesShaped(const FrameJob &J, int s);

static int stageTiles(const FrameJob &J, int s, const LaunchConfig &cfg) {
    if (stageTunable(s)) {
        const int base = stageTilesShaped(J, s);
        if (base == 0) return 0;
        const int bx = cfg.shapeX[s], by = cfg.shapeY[s];
        switch (s) {
        case S_DET_TRANSFER: case S_BM_AGG: return cdiv(J.W, bx) * cdiv(J.H, by);
        case S_HPASS: return cdiv(J.W, bx) * cdiv(J.ch, by);
        case S_AFFINE: case S_LGF_DENSE: case S_YC: return cdiv(J.cw, bx) * cdiv(J.ch, by);
        case S_DET_PLAIN: return cdiv(J.sw, bx) * cdiv(J.sh, by);
        }
    }
    return stageTilesShaped(J, s);
}

static int stageTilesShaped(const FrameJob &J, int s) {
    const bool resize = !J.sameSize;
    if (s >= S_NYQ0 && s <= S_NYQ7) {
        const int pass = s - S_NYQ0;
        return (J.guided && J.algo == 6 && !J.detailFused && pass < J.nyqX + J.nyqY) ? cdiv(J.sw, 32) * cdiv(J.sh, 8) : 0;
    }
    switch (s) {
    case S_CONVERT: return convertLumaBlocks(J.sw, J.sh) + convertBlocks(J.cw, J.ch);
    case S_LUMA_RADIAL: return (resize && J.writeLuma && J.radial) ? cdiv(J.W, 32) * cdiv(J.H, 32) : 0;
    case S_LUMA_H: return (resize && J.writeLuma && !J.radial) ? cdiv(J.W, 32) * cdiv(J.sh, 8) : 0;
    case S_LUMA_V: return (resize && J.writeLuma && !J.radial) ? cdiv(J.W, 32) * cdiv(J.H, 8) : 0;
    case S_TENSOR: return J.guided ? cdiv(J.sw, kTensorCols * kTensorWarps) * cdiv(J.sh, kTensorRows) : 0;
    case S_DIL_H: return J.sparse ? J.sh : 0;
    case S_DIL_V: return J.sparse ? cdiv(J.maskWords, 32) * cdiv(J.sh, 8) : 0;
    case S_MARK: {
        const int g = std::max(1, J.listGroup);
        return (J.sparse || J.listed) ? cdiv(cdiv(J.H, g) * g * cdiv(J.W, 32), 256) : 0;
    }
    case S_COUNT: return J.sparse ? cdiv(J.cw * J.ch, kCountChunk) : 0;
    case S_GATE: return J.useMs ? cdiv(J.cw, 32) * cdiv(J.ch, kGateRows) : 0;
    case S_LGF_DENSE: return (J.guided && J.algo == 4 && !J.lgfRoiOnly) ? cdiv(J.cw, 32) * cdiv(J.ch, 8) : 0;
    case S_HPASS: return (J.hTab && !J.radial && !J.plainFused && (J.kernel != 0 || J.guided)) ? cdiv(J.W, 32) * cdiv(J.ch, 8) : 0;
    case S_PLAIN: return cdiv(J.W, 32) * cdiv(J.H, J.plainRows);
    case S_GUIDED: return J.listed ? 1 : 0;
    case S_YC: return (J.guided && J.algo == 6 && !J.ycTiled) ? cdiv(J.cw, 32) * cdiv(J.ch, 8) : 0;
    case S_YC_TILED: return (J.guided && J.algo == 6 && J.ycTiled) ? cdiv(J.cw, kYcTile) * cdiv(J.ch, kYcTile) : 0;
    case S_AFFINE: return (J.guided && J.algo == 6 && !J.chromaList) ? cdiv(J.cw, 32) * cdiv(J.ch, 8) : 0;
    case S_AFFINE_LIST: return J.chromaList ? 1 : 0;
    case S_DET_HPASS: return (J.guided && J.algo == 6 && J.dTab && !J.detailFused) ? cdiv(J.sw, 32) * cdiv(J.ch, 8) : 0;
    case S_DET_PLAIN: return (J.guided && J.algo == 6 && !J.detailFused) ? cdiv(J.sw, 32) * cdiv(J.sh, 8) : 0;
    case S_DET_MAP: return (J.guided && J.algo == 6 && J.detailFused) ? cdiv(J.sw, kDetailTile) * cdiv(J.sh, J.detailRows) : 0;
    case S_DET_RH: return (J.guided && J.algo == 6 && resize && !J.radial) ? cdiv(J.W, 32) * cdiv(J.sh, 8) : 0;
    case S_DET_RV: return (J.guided && J.algo == 6 && resize && !J.radial) ? cdiv(J.W, 32) * cdiv(J.H, 8) : 0;
    case S_DET_RR: return (J.guided && J.algo == 6 && resize && J.radial) ? cdiv(J.W, 32) * cdiv(J.H, 8) : 0;
    case S_DET_TRANSFER: return (J.guided && J.algo == 6 && !J.xferListed) ? cdiv(J.W, 32) * cdiv(J.H, 8) : 0;
    case S_DET_XFER_LIST: return J.xferListed ? 1 : 0;
    case S_ROI:
    case S_BLEND: return (J.guided && J.algo == 4 && J.lgfRoiOnly) ? cdiv(J.W, 32) * cdiv(J.H, 8) : 0;
    case S_BM_GROUP: return J.bm ? cdiv(J.bmAnchorsX * J.bmAnchorsY, 8) : 0;
    case S_BM_AGG: return J.bm ? cdiv(J.W, 32) * cdiv(J.H, 8) : 0;
    case S_BP: return J.needBackProject ? cdiv(J.cw, 32) * cdiv(J.ch, 8) : 0;
    case S_LGF_ROI: return (J.guided && J.algo == 4 && J.lgfRoiOnly) ? cdiv(J.cw, 32) * cdiv(J.ch, 8) : 0;
    case S_STORE: return (J.directOutput || J.finalInTransfer || J.blendStores || J.bpStores) ? 0 : cdiv(J.W, 32) * cdiv(J.H, 8);
    }
    return 0;
}

void planStages(const std::vector<FrameJob> &jobs, StagePlan &plan, const LaunchConfig *cfg) {
    const int n = int(jobs.size());
    plan.cfg = cfg ? *cfg : processLaunchConfig();
    plan.prefix.assign(size_t(S_N) * (n + 1), 0);
    plan.totals.assign(S_N, 0);
    plan.maxDil = 0;
    for (int s = 0; s < S_N; ++s) {
        int acc = 0;
        for (int f = 0; f < n; ++f) {
            plan.prefix[size_t(s) * (n + 1) + f] = acc;
            acc += stageTiles(jobs[f], s, plan.cfg);
        }
        plan.prefix[size_t(s) * (n + 1) + n] = acc;
        plan.totals[s] = acc;
    }
    for (const FrameJob &J : jobs)
        if (J.sparse)
            plan.maxDil = std::max(plan.maxDil, J.dil);
}

int launchStages(const std::vector<FrameJob> &jobs, const StagePlan &plan, const FrameJob *dJobs,
                 const int *dPrefix, cudaStream_t stream) {
    const int n = int(jobs.size());
    int launches = 0;
    const dim3 b32x8(32, 8);
    auto pre = [&](int s) { return dPrefix + size_t(s) * (n + 1); };
    auto go = [&](int s, auto kernel, dim3 block, size_t smem = 0) {
        if (plan.totals[s] == 0)
            return;
        if (stageTunable(s))
            block = dim3(plan.cfg.shapeX[s], plan.cfg.shapeY[s]);
        kernel<<<plan.totals[s], block, smem, stream>>>(dJobs, pre(s), n);
        ++launches;
    };
    go(S_CONVERT, k_convert, dim3(kConvertWarps * 32));
    go(S_LUMA_RADIAL, k_luma_radial, b32x8);
    go(S_LUMA_H, k_luma_h, b32x8);
    go(S_LUMA_V, k_luma_v, b32x8);
    go(S_TENSOR, k_tensor, dim3(kTensorWarps * 32));
    go(S_DIL_H, k_dilate_h, dim3(128));
    go(S_DIL_V, k_dilate_v, dim3(32, 8));
    go(S_MARK, k_mark_chroma, dim3(256));
    go(S_COUNT, k_count, dim3(256));
    go(S_GATE, k_gate, b32x8);
    go(S_LGF_DENSE, k_lgf, b32x8);
    go(S_HPASS, k_hpass, b32x8);
    // jinc selector frames in this launch: the plain and guided instances
    // that know the guided pass forms their plain base
    bool rfuse = false, ronly = !jobs.empty();
    for (const FrameJob &J : jobs) {
        rfuse = rfuse || radialPlainFused(J);
        ronly = ronly && radialPlainFused(J);
    }
    if (plan.totals[S_PLAIN] > 0) {
        // the dynamic shared-memory opt-in is per device (idempotent, so a
        // race between host threads only repeats it)
        static std::atomic<int> plainOptIn[64];
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64 || !plainOptIn[dev].load()) {
            cudaFuncSetAttribute(k_plain, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kPlainDynSmem));
            cudaFuncSetAttribute(k_plain_all, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(kPlainDynSmem));
            if (dev >= 0 && dev < 64)
                plainOptIn[dev].store(1);
        }
    }
    if (rfuse)
        go(S_PLAIN, k_plain_all, b32x8, kPlainDynSmem);
    else
        go(S_PLAIN, k_plain, b32x8, kPlainDynSmem);
    if (plan.totals[S_GUIDED] > 0) {
        // persistent grid: enough resident blocks to fill every SM
        const int variant = plan.cfg.guidedVariant;
        // the instance with the fused jinc plain base when a frame needs it
        using GuidedKernel = void (*)(const FrameJob *, const int *, int);
        static const GuidedKernel kernelsOf[3][3] = {
            {k_guided, k_guided3, k_guided_staged}, {k_guided_r, k_guided3_r, k_guided_staged_r},
            {k_guided_o, k_guided3_o, k_guided_staged_o}};
        const int inst = ronly ? 2 : rfuse ? 1 : 0;
        const GuidedKernel kern = kernelsOf[inst][variant];
        static int gridBlocks[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const size_t dyn = variant == 2 ? kGuidedStageBytes : 0;
        int &grid = gridBlocks[inst][variant];
        if (grid == 0) {
            int dev = 0, sms = 0, perSm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (variant == 2)
                cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(kGuidedStageBytes));
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, 256, dyn);
            grid = std::max(1, sms * std::max(1, perSm));
        }
        kern<<<grid, 256, dyn, stream>>>(dJobs, pre(S_GUIDED), n);
        ++launches;
    }
    go(S_YC, k_yc_h, b32x8);
    go(S_YC_TILED, k_yc_tiled, b32x8);
    go(S_AFFINE, k_affine, b32x8);
    if (plan.totals[S_AFFINE_LIST] > 0) {
        // persistent grid over the algo 6 frames' chroma lists
        static int gridBlocks = 0;
        if (gridBlocks == 0) {
            int dev = 0, sms = 0, perSm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_affine_list, 256, 0);
            gridBlocks = std::max(1, sms * std::max(1, perSm));
        }
        k_affine_list<<<gridBlocks, 256, 0, stream>>>(dJobs, pre(S_AFFINE_LIST), n);
        ++launches;
    }
    go(S_DET_HPASS, k_detail_hpass, b32x8);
    go(S_DET_PLAIN, k_detail_plain, b32x8);
    go(S_DET_MAP, k_detail_map, b32x8);
    for (int pass = 0; pass < 8; ++pass) {
        const int s = S_NYQ0 + pass;
        if (plan.totals[s] == 0)
            continue;
        k_detail_nyq<<<plan.totals[s], b32x8, 0, stream>>>(dJobs, pre(s), n, pass);
        ++launches;
    }
    go(S_DET_RH, k_detail_resize_h, b32x8);
    go(S_DET_RV, k_detail_resize_v, b32x8);
    go(S_DET_RR, k_detail_resize_radial, b32x8);
    go(S_DET_TRANSFER, k_detail_transfer, b32x8);
    if (plan.totals[S_DET_XFER_LIST] > 0) {
        // persistent grid over the algo 6 frames' work lists
        static int gridBlocks = 0;
        if (gridBlocks == 0) {
            int dev = 0, sms = 0, perSm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_detail_transfer_list, 256, 0);
            gridBlocks = std::max(1, sms * std::max(1, perSm));
        }
        k_detail_transfer_list<<<gridBlocks, 256, 0, stream>>>(dJobs, pre(S_DET_XFER_LIST), n);
        ++launches;
    }
    go(S_ROI, k_roi, b32x8);
    go(S_LGF_ROI, k_lgf, b32x8);
    go(S_BLEND, k_blend, b32x8);
    go(S_BM_GROUP, k_bm_group, dim3(256));
    go(S_BM_AGG, k_bm_aggregate, b32x8);
    go(S_BP, k_backproject, b32x8);
    go(S_STORE, k_store_chroma, b32x8);
    if (cudaPeekAtLastError() != cudaSuccess)
        return -1;
    return launches;
}

} // namespace lgcr_b200
