// C ABI of the Downsample filter (include/lgcr_b200.h): downsampleCreate /
// downsampleGetFrame / downsampleFree (src/downsample.cpp:740-918) over the
// device kernels of kernels_downsample.cu.
//
// The polyphase tables of the base are built once at create time for the
// clip's constant size (buildDownsampleWeights, downsample.cpp:52-93) and
// stay resident. Each call takes a workspace from a small pool (the
// horizontal-pass rows, the quality-2 candidate planes, host-path staging),
// so calls from several host threads are safe.
#include "impl.h"
#include "downsample.h"
#include "geometry.h"

#include <cmath>
#include <cstring>

using namespace lgcr_b200;

namespace {

enum DsKernel : int { kDsSpline36 = 0, kDsLanczos3 = 1, kDsBinomial = 2 };

// buildBinomialWeights (downsample.cpp:52-84): [1 4 6 4 1]/16 centred on the
// nearest sample when the phase is a whole sample, else [1 3 3 1]/8
WeightTable binomialWeights(int srcN, float shift) {
    WeightTable t;
    t.n = srcN / 2;
    const bool integerPhase = std::fabs(std::fabs(shift) - 0.5f) < 1e-6f;
    t.sup = integerPhase ? 5 : 4;
    t.start.resize(t.n);
    t.w.resize(size_t(t.n) * t.sup);
    static const float whole[5] = {1.0f / 16.0f, 4.0f / 16.0f, 6.0f / 16.0f, 4.0f / 16.0f, 1.0f / 16.0f};
    static const float half[4] = {1.0f / 8.0f, 3.0f / 8.0f, 3.0f / 8.0f, 1.0f / 8.0f};
    for (int i = 0; i < t.n; ++i) {
        const float center = 2.0f * i + 0.5f + shift;
        if (integerPhase) {
            t.start[i] = int(std::lround(center)) - 2;
            std::memcpy(&t.w[size_t(i) * 5], whole, sizeof(whole));
        } else {
            t.start[i] = int(std::floor(center)) - 1;
            std::memcpy(&t.w[size_t(i) * 4], half, sizeof(half));
        }
    }
    return t;
}

WeightTable downsampleWeights(int srcN, int kernel, float shift) {
    if (kernel == kDsBinomial)
        return binomialWeights(srcN, shift);
    KernelSpec k;
    k.kernel = kernel == kDsSpline36 ? Kernel::Spline36 : Kernel::Lanczos;
    k.kp1 = 3.0;
    k.kp2 = 0.0;
    k.support = 3.0;
    return buildWeights(srcN, srcN / 2, k, shift);
}

struct DsWorkspace {
    DeviceArena arena;
    float2 *rows = nullptr;
    float *cand = nullptr;
    void *stageIn[3] = {nullptr, nullptr, nullptr};
    void *stageOut[2] = {nullptr, nullptr};
    bool host = false;
    cudaEvent_t done = nullptr;
    bool used = false;
    ~DsWorkspace() {
        if (done) cudaEventDestroy(done);
    }
};

} // namespace

struct lgcr_downsample {
    lgcr_format fmt{};
    int quality = 0, kernel = kDsSpline36, chromaLocation = 0;
    float strength = 1.0f, shiftX = -0.5f, shiftY = 0.0f;
    DeviceArena tables;
    int hSup = 0, vSup = 0;
    const int *hStart = nullptr, *vStart = nullptr;
    const float *hW = nullptr, *vW = nullptr;
    std::mutex mu;
    std::vector<std::unique_ptr<DsWorkspace>> idle;

    int bps() const { return fmt.sample_type == LGCR_ST_FLOAT ? 4 : (fmt.bits_per_sample > 8 ? 2 : 1); }
    bool candidates() const { return quality == 2 && strength != 0.0f; }

    DsWorkspace *acquire(bool host) {
        {
            std::lock_guard<std::mutex> lock(mu);
            for (size_t i = 0; i < idle.size(); ++i)
                if (!host || idle[i]->host) {
                    DsWorkspace *w = idle[i].release();
                    idle.erase(idle.begin() + i);
                    return w;
                }
        }
        const int W = fmt.width, H = fmt.height, cw = W / 2, ch = H / 2;
        auto w = std::make_unique<DsWorkspace>();
        const size_t oRows = w->arena.reserve(size_t(H) * cw * sizeof(float2));
        const size_t oCand = candidates() ? w->arena.reserve(size_t(kDsPlanes) * cw * ch * 4) : 0;
        size_t oIn[3] = {0, 0, 0}, oOut[2] = {0, 0};
        if (host) {
            for (int p = 0; p < 3; ++p)
                oIn[p] = w->arena.reserve(size_t(W) * H * bps());
            for (int p = 0; p < 2; ++p)
                oOut[p] = w->arena.reserve(size_t(cw) * ch * bps());
        }
        if (!w->arena.commit() ||
            cudaEventCreateWithFlags(&w->done, cudaEventDisableTiming) != cudaSuccess)
            return nullptr;
        w->rows = (float2 *)w->arena.at(oRows);
        w->cand = candidates() ? (float *)w->arena.at(oCand) : nullptr;
        w->host = host;
        if (host) {
            for (int p = 0; p < 3; ++p)
                w->stageIn[p] = w->arena.at(oIn[p]);
            for (int p = 0; p < 2; ++p)
                w->stageOut[p] = w->arena.at(oOut[p]);
        }
        return w.release();
    }

    void release(DsWorkspace *w) {
        std::lock_guard<std::mutex> lock(mu);
        idle.emplace_back(w);
        if (idle.size() > 8)
            idle.erase(idle.begin());
    }
};

extern "C" {

void lgcr_downsample_params_init(lgcr_downsample_params *p) {
    if (!p)
        return;
    p->quality = LGCR_UNSET_INT;
    p->kernel = nullptr;
    p->strength = 1.0;
    p->strength_set = 0;
    p->loc = nullptr;
}

int lgcr_downsample_create(const lgcr_downsample_params *params, const lgcr_format *fmt,
                           lgcr_downsample **out, char *err, size_t errlen) {
    auto fail = [&](const char *msg, int code = LGCR_E_INVALID) {
        setError(msg);
        if (err && errlen) {
            std::strncpy(err, msg, errlen - 1);
            err[errlen - 1] = '\0';
        }
        return code;
    };
    if (!fmt || !out)
        return fail("Downsample: null argument", LGCR_E_ARGUMENT);
    // downsampleCreate src/downsample.cpp:830-846
    const bool integerFormat = fmt->sample_type == LGCR_ST_INTEGER && fmt->bits_per_sample >= 8 &&
                               fmt->bits_per_sample <= 16;
    const bool floatFormat = fmt->sample_type == LGCR_ST_FLOAT && fmt->bits_per_sample == 32;
    if (fmt->color_family != LGCR_CF_YUV || fmt->subsampling_w != 0 || fmt->subsampling_h != 0 ||
        (!integerFormat && !floatFormat))
        return fail("Downsample: input must be planar YUV444 (8-16 bit integer or float32)");
    if (fmt->width <= 0 || fmt->height <= 0 || (fmt->width & 1) != 0 || (fmt->height & 1) != 0)
        return fail("Downsample: constant even input width and height are required");
    auto d = std::make_unique<lgcr_downsample>();
    d->fmt = *fmt;
    const lgcr_downsample_params none = {LGCR_UNSET_INT, nullptr, 1.0, 0, nullptr};
    const lgcr_downsample_params &p = params ? *params : none;
    d->quality = p.quality == LGCR_UNSET_INT ? 0 : p.quality;
    if (d->quality < 0 || d->quality > 2)
        return fail("Downsample: quality must be 0, 1, or 2");
    const std::string kernel = p.kernel ? p.kernel : "spline36";
    if (kernel == "spline36")
        d->kernel = kDsSpline36;
    else if (kernel == "lanczos3")
        d->kernel = kDsLanczos3;
    else if (kernel == "binomial")
        d->kernel = kDsBinomial;
    else
        return fail("Downsample: kernel must be \"spline36\", \"lanczos3\", or \"binomial\"");
    d->strength = p.strength_set ? float(p.strength) : 1.0f;
    if (!std::isfinite(d->strength) || d->strength < 0.0f || d->strength > 1.0f)
        return fail("Downsample: strength must be in the range 0..1");
    // loc -> (shiftX, shiftY, _ChromaLocation), src/downsample.cpp:880-899
    static const struct { const char *name; float sx, sy; int cl; } sitings[6] = {
        {"left", -0.5f, 0.0f, 0}, {"center", 0.0f, 0.0f, 1}, {"topleft", -0.5f, -0.5f, 2},
        {"top", 0.0f, -0.5f, 3}, {"bottomleft", -0.5f, 0.5f, 4}, {"bottom", 0.0f, 0.5f, 5}};
    const std::string loc = p.loc ? p.loc : "left";
    int which = -1;
    for (int i = 0; i < 6; ++i)
        if (loc == sitings[i].name)
            which = i;
    if (which < 0)
        return fail("Downsample: loc must be left, center, topleft, top, bottomleft, or bottom");
    d->shiftX = sitings[which].sx;
    d->shiftY = sitings[which].sy;
    d->chromaLocation = sitings[which].cl;

    const WeightTable tx = downsampleWeights(fmt->width, d->kernel, d->shiftX);
    const WeightTable ty = downsampleWeights(fmt->height, d->kernel, d->shiftY);
    const size_t oHs = d->tables.reserve(tx.start.size() * 4), oHw = d->tables.reserve(tx.w.size() * 4);
    const size_t oVs = d->tables.reserve(ty.start.size() * 4), oVw = d->tables.reserve(ty.w.size() * 4);
    if (!d->tables.commit())
        return fail("Downsample: device table allocation failed", LGCR_E_NOMEM);
    const struct { size_t off; const void *src; size_t bytes; } up[4] = {
        {oHs, tx.start.data(), tx.start.size() * 4}, {oHw, tx.w.data(), tx.w.size() * 4},
        {oVs, ty.start.data(), ty.start.size() * 4}, {oVw, ty.w.data(), ty.w.size() * 4}};
    for (const auto &u : up)
        if (cudaMemcpy(d->tables.at(u.off), u.src, u.bytes, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail("Downsample: table upload failed", LGCR_E_CUDA);
    d->hSup = tx.sup;
    d->vSup = ty.sup;
    d->hStart = (const int *)d->tables.at(oHs);
    d->hW = (const float *)d->tables.at(oHw);
    d->vStart = (const int *)d->tables.at(oVs);
    d->vW = (const float *)d->tables.at(oVw);
    *out = d.release();
    return LGCR_OK;
}

void lgcr_downsample_destroy(lgcr_downsample *d) {
    if (!d)
        return;
    cudaDeviceSynchronize();
    delete d;
}

int lgcr_downsample_chroma_location(const lgcr_downsample *d) { return d ? d->chromaLocation : -1; }

int lgcr_downsample_frame(lgcr_downsample *d, const lgcr_plane in[3], const lgcr_plane out[3],
                          int memory, void *stream) {
    if (!d || !in || !out) {
        setError("Downsample: null argument");
        return LGCR_E_ARGUMENT;
    }
    const int bps = d->bps();
    const int W = d->fmt.width, H = d->fmt.height, cw = W / 2, ch = H / 2;
    bool ok = true;
    for (int p = 0; p < 3 && ok; ++p)
        ok = in[p].data && in[p].width == W && in[p].height == H &&
             in[p].stride >= (ptrdiff_t)W * bps;
    for (int p = 1; p < 3 && ok; ++p)
        ok = out[p].data && out[p].width == cw && out[p].height == ch &&
             out[p].stride >= (ptrdiff_t)cw * bps;
    if (ok && out[0].data)
        ok = out[0].width == W && out[0].height == H && out[0].stride >= (ptrdiff_t)W * bps;
    if (!ok) {
        setError("Downsample: plane dimensions or strides do not match the clip format");
        return LGCR_E_ARGUMENT;
    }
    if (memory != LGCR_MEM_HOST && memory != LGCR_MEM_DEVICE) {
        setError("Downsample: memory must be LGCR_MEM_HOST or LGCR_MEM_DEVICE");
        return LGCR_E_ARGUMENT;
    }
    const bool host = memory == LGCR_MEM_HOST;
    DsWorkspace *ws = d->acquire(host);
    if (!ws) {
        setError("Downsample: device workspace allocation failed");
        return LGCR_E_NOMEM;
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : (host ? callingThreadStream() : nullptr);
    cudaError_t e = ws->used ? cudaStreamWaitEvent(st, ws->done, 0) : cudaSuccess;

    DownsampleJob J;
    std::memset(&J, 0, sizeof(J));
    J.W = W; J.H = H; J.cw = cw; J.ch = ch;
    const bool isFloat = d->fmt.sample_type == LGCR_ST_FLOAT;
    J.kind = isFloat ? kF32 : (bps == 2 ? kU16 : kU8);
    // processFrame's SourcePlane / OutputPlane constants (downsample.cpp:656-679)
    const int maxValue = isFloat ? 0 : (1 << d->fmt.bits_per_sample) - 1;
    J.inScale = isFloat ? 1.0f : 1.0f / maxValue;
    J.chromaOffset = isFloat ? 0.0f : -0.5f;
    J.outScale = float(maxValue);
    J.outOffset = 0.5f * J.outScale;
    J.maxCode = maxValue;
    for (int p = 0; p < 3; ++p) {
        if (host) {
            if (e == cudaSuccess)
                e = copyPlane(ws->stageIn[p], size_t(W) * bps, in[p].data, in[p].stride,
                              size_t(W) * bps, H, cudaMemcpyHostToDevice, st);
            J.in[p] = ws->stageIn[p];
            J.inPitch[p] = (long long)W * bps;
        } else {
            J.in[p] = in[p].data;
            J.inPitch[p] = in[p].stride;
        }
    }
    for (int p = 0; p < 2; ++p) {
        J.out[p] = host ? ws->stageOut[p] : out[p + 1].data;
        J.outPitch[p] = host ? (long long)cw * bps : (long long)out[p + 1].stride;
    }
    J.hSup = d->hSup; J.vSup = d->vSup;
    J.hStart = d->hStart; J.vStart = d->vStart;
    J.hW = d->hW; J.vW = d->vW;
    J.rows = ws->rows;
    J.cand = ws->cand;
    J.quality = d->quality;
    J.strength = d->strength;
    J.shiftX = d->shiftX;
    J.shiftY = d->shiftY;
    if (e == cudaSuccess)
        e = launchDownsample(J, st);
    // luma: the reference shares the source's Y plane with its output frame
    if (e == cudaSuccess && out[0].data && !host)
        e = cudaMemcpy2DAsync(out[0].data, out[0].stride, in[0].data, in[0].stride,
                              size_t(W) * bps, H, cudaMemcpyDeviceToDevice, st);
    if (host)
        for (int p = 0; p < 2 && e == cudaSuccess; ++p)
            e = copyPlane(out[p + 1].data, out[p + 1].stride, ws->stageOut[p], size_t(cw) * bps,
                          size_t(cw) * bps, ch, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaEventRecord(ws->done, st);
    ws->used = true;
    d->release(ws);
    if (e == cudaSuccess && host) {
        e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && out[0].data)
            for (int y = 0; y < H; ++y)
                std::memcpy(static_cast<char *>(out[0].data) + (ptrdiff_t)y * out[0].stride,
                            static_cast<const char *>(in[0].data) + (ptrdiff_t)y * in[0].stride,
                            size_t(W) * bps);
    }
    if (e != cudaSuccess)
        return cudaFail(e, "lgcr_downsample_frame");
    return LGCR_OK;
}

} // extern "C"
