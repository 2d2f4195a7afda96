// C ABI of the Sharpen filter (include/lgcr_b200.h): sharpenCreate /
// sharpenGetFrame / sharpenFree (src/plugin.cpp:14-111) over device kernels.
//
// A filter keeps, per frame size, the footprint tables of its chroma guide
// and a small pool of workspaces (the float sharpened-luma plane the chroma
// pass reads, plus host-path staging planes). Calls from several host
// threads are safe; each call takes its own workspace.
#include "impl.h"
#include "sharpen.h"

#include <cmath>
#include <cstring>

using namespace lgcr_b200;

namespace {

struct SharpenSize {
    int sw = 0, sh = 0, cw = 0, ch = 0;
    DeviceArena tables;                 // lcXb, lcXe, lcYb, lcYe
    const int *lcXb = nullptr, *lcXe = nullptr, *lcYb = nullptr, *lcYe = nullptr;
};

struct SharpenWorkspace {
    int sw = 0, sh = 0;
    DeviceArena arena;
    float *Ys = nullptr;
    void *stageIn[3] = {nullptr, nullptr, nullptr}, *stageOut[3] = {nullptr, nullptr, nullptr};
    size_t pitch[3] = {0, 0, 0};
    cudaEvent_t done = nullptr;
    bool used = false;
    ~SharpenWorkspace() {
        if (done) cudaEventDestroy(done);
    }
};

} // namespace

struct lgcr_sharpen {
    lgcr_format fmt{};
    double alpha = 0.3, sigma = 0.01, sratio = 0.15, gspatial = 1.2, ar = 0.0;
    std::mutex mu;
    std::vector<std::unique_ptr<SharpenSize>> sizes;
    std::vector<std::unique_ptr<SharpenWorkspace>> idle;

    int bps() const { return fmt.sample_type == LGCR_ST_FLOAT ? 4 : (fmt.bits_per_sample > 8 ? 2 : 1); }

    const SharpenSize *sizeFor(int sw, int sh, int cw, int ch) {
        std::lock_guard<std::mutex> lock(mu);
        for (auto &s : sizes)
            if (s->sw == sw && s->sh == sh && s->cw == cw && s->ch == ch)
                return s.get();
        auto s = std::make_unique<SharpenSize>();
        s->sw = sw; s->sh = sh; s->cw = cw; s->ch = ch;
        // left siting on subsampled axes, as the reference's Sharpen hard-codes
        const double rw = double(sw) / cw, rh = double(sh) / ch;
        std::vector<int> xb, xe, yb, ye;
        lcExtents(sw, cw, rw, -0.5, xb, xe);
        lcExtents(sh, ch, rh, 0.0, yb, ye);
        const size_t oxb = s->tables.reserve(xb.size() * 4), oxe = s->tables.reserve(xe.size() * 4);
        const size_t oyb = s->tables.reserve(yb.size() * 4), oye = s->tables.reserve(ye.size() * 4);
        if (!s->tables.commit())
            return nullptr;
        const std::pair<size_t, const std::vector<int> *> parts[4] = {
            {oxb, &xb}, {oxe, &xe}, {oyb, &yb}, {oye, &ye}};
        for (const auto &pt : parts)
            if (cudaMemcpy(s->tables.at(pt.first), pt.second->data(), pt.second->size() * 4,
                           cudaMemcpyHostToDevice) != cudaSuccess)
                return nullptr;
        s->lcXb = (const int *)s->tables.at(oxb); s->lcXe = (const int *)s->tables.at(oxe);
        s->lcYb = (const int *)s->tables.at(oyb); s->lcYe = (const int *)s->tables.at(oye);
        sizes.push_back(std::move(s));
        return sizes.back().get();
    }

    SharpenWorkspace *acquire(int sw, int sh, int cw, int ch, bool host) {
        {
            std::lock_guard<std::mutex> lock(mu);
            for (size_t i = 0; i < idle.size(); ++i)
                if (idle[i]->sw == sw && idle[i]->sh == sh &&
                    (!host || idle[i]->stageIn[0] != nullptr)) {
                    SharpenWorkspace *w = idle[i].release();
                    idle.erase(idle.begin() + i);
                    return w;
                }
        }
        auto w = std::make_unique<SharpenWorkspace>();
        w->sw = sw; w->sh = sh;
        const size_t oY = w->arena.reserve(size_t(sw) * sh * 4);
        size_t oIn[3] = {0, 0, 0}, oOut[3] = {0, 0, 0};
        if (host) {
            for (int p = 0; p < 3; ++p) {
                const int pw = p ? cw : sw, ph = p ? ch : sh;
                w->pitch[p] = size_t(pw) * bps();
                oIn[p] = w->arena.reserve(w->pitch[p] * ph);
                oOut[p] = w->arena.reserve(w->pitch[p] * ph);
            }
        }
        if (!w->arena.commit() ||
            cudaEventCreateWithFlags(&w->done, cudaEventDisableTiming) != cudaSuccess)
            return nullptr;
        w->Ys = (float *)w->arena.at(oY);
        if (host)
            for (int p = 0; p < 3; ++p) {
                w->stageIn[p] = w->arena.at(oIn[p]);
                w->stageOut[p] = w->arena.at(oOut[p]);
            }
        return w.release();
    }

    void release(SharpenWorkspace *w) {
        std::lock_guard<std::mutex> lock(mu);
        idle.emplace_back(w);
        if (idle.size() > 8)
            idle.erase(idle.begin());
    }
};

extern "C" {

void lgcr_sharpen_params_init(lgcr_sharpen_params *p) {
    if (!p)
        return;
    p->alpha = p->sigma = p->sratio = p->gspatial = p->ar = NAN;
}

int lgcr_sharpen_create(const lgcr_sharpen_params *params, const lgcr_format *fmt,
                        lgcr_sharpen **out, char *err, size_t errlen) {
    auto fail = [&](const char *msg) {
        setError(msg);
        if (err && errlen) {
            std::strncpy(err, msg, errlen - 1);
            err[errlen - 1] = '\0';
        }
        return LGCR_E_INVALID;
    };
    if (!fmt || !out)
        return fail("LGCR Sharpen: null argument");
    // sharpenCreate src/plugin.cpp:90-103
    if (fmt->color_family != LGCR_CF_YUV ||
        (fmt->sample_type == LGCR_ST_FLOAT && fmt->bits_per_sample != 32) ||
        (fmt->sample_type != LGCR_ST_FLOAT &&
         (fmt->bits_per_sample < 8 || fmt->bits_per_sample > 16)))
        return fail("LGCR Sharpen: planar YUV only");
    auto s = std::make_unique<lgcr_sharpen>();
    s->fmt = *fmt;
    if (params) {
        if (!std::isnan(params->alpha)) s->alpha = params->alpha;
        if (!std::isnan(params->sigma)) s->sigma = params->sigma;
        if (!std::isnan(params->sratio)) s->sratio = params->sratio;
        if (!std::isnan(params->gspatial)) s->gspatial = params->gspatial;
        if (!std::isnan(params->ar)) s->ar = params->ar;
    }
    if (s->sigma <= 0.0 || s->sratio <= 0.0 || s->gspatial <= 0.0)
        return fail("LGCR Sharpen: sigma/sratio/gspatial must be > 0");
    *out = s.release();
    return LGCR_OK;
}

void lgcr_sharpen_destroy(lgcr_sharpen *s) {
    if (!s)
        return;
    cudaDeviceSynchronize();
    delete s;
}

int lgcr_sharpen_frame(lgcr_sharpen *s, const lgcr_plane in[3], const lgcr_plane out[3],
                       int memory, void *stream) {
    if (!s || !in || !out) {
        setError("LGCR Sharpen: null argument");
        return LGCR_E_ARGUMENT;
    }
    const int bps = s->bps();
    const int sw = in[0].width, sh = in[0].height;
    const int cw = in[1].width, ch = in[1].height;
    const int ssw = s->fmt.subsampling_w, ssh = s->fmt.subsampling_h;
    bool ok = sw > 0 && sh > 0 && ssw >= 0 && ssh >= 0 && ssw < 8 && ssh < 8 &&
              cw == ((sw + (1 << ssw) - 1) >> ssw) && ch == ((sh + (1 << ssh) - 1) >> ssh) &&
              in[2].width == cw && in[2].height == ch &&
              (s->fmt.width == 0 || (s->fmt.width == sw && s->fmt.height == sh));
    for (int p = 0; p < 3 && ok; ++p) {
        const int pw = p ? cw : sw, ph = p ? ch : sh;
        ok = in[p].data && out[p].data && in[p].stride >= (ptrdiff_t)pw * bps &&
             out[p].width == pw && out[p].height == ph && out[p].stride >= (ptrdiff_t)pw * bps;
    }
    if (!ok) {
        setError("LGCR Sharpen: plane dimensions or strides do not match the clip format");
        return LGCR_E_ARGUMENT;
    }
    if (memory != LGCR_MEM_HOST && memory != LGCR_MEM_DEVICE) {
        setError("LGCR Sharpen: memory must be LGCR_MEM_HOST or LGCR_MEM_DEVICE");
        return LGCR_E_ARGUMENT;
    }
    const bool host = memory == LGCR_MEM_HOST;
    const bool guided = cw != sw || ch != sh;
    const SharpenSize *sz = guided ? s->sizeFor(sw, sh, cw, ch) : nullptr;
    if (guided && !sz) {
        setError("LGCR Sharpen: failed to upload the footprint tables");
        return LGCR_E_NOMEM;
    }
    SharpenWorkspace *ws = s->acquire(sw, sh, cw, ch, host);
    if (!ws) {
        setError("LGCR Sharpen: device workspace allocation failed");
        return LGCR_E_NOMEM;
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : (host ? callingThreadStream() : nullptr);
    cudaError_t e = ws->used ? cudaStreamWaitEvent(st, ws->done, 0) : cudaSuccess;

    SharpenJob J;
    std::memset(&J, 0, sizeof(J));
    J.sw = sw; J.sh = sh; J.cw = cw; J.ch = ch;
    const bool isFloat = s->fmt.sample_type == LGCR_ST_FLOAT;
    J.kind = isFloat ? kF32 : (bps == 2 ? kU16 : kU8);
    const int bits = s->fmt.bits_per_sample;
    J.yScale = isFloat ? 1.0 : 1.0 / double((1 << bits) - 1);
    J.cOffset = isFloat ? 0.0 : -0.5;
    const double outScale = isFloat ? 1.0 : double((1 << bits) - 1);
    J.qScale = float(outScale);
    J.qOffC = float(isFloat ? 0.0 : 0.5 * outScale);
    J.maxCode = isFloat ? 0 : (1 << bits) - 1;
    for (int p = 0; p < 3; ++p) {
        const int pw = p ? cw : sw, ph = p ? ch : sh;
        if (host) {
            if (e == cudaSuccess)
                e = copyPlane(ws->stageIn[p], ws->pitch[p], in[p].data, in[p].stride,
                              size_t(pw) * bps, ph, cudaMemcpyHostToDevice, st);
            J.in[p] = ws->stageIn[p];
            J.inPitch[p] = (long long)ws->pitch[p];
            J.out[p] = ws->stageOut[p];
            J.outPitch[p] = (long long)ws->pitch[p];
        } else {
            J.in[p] = in[p].data;
            J.inPitch[p] = in[p].stride;
            J.out[p] = out[p].data;
            J.outPitch[p] = out[p].stride;
        }
    }
    J.Ys = guided ? ws->Ys : nullptr;
    J.alpha = float(s->alpha);
    J.sigma = float(s->sigma);
    J.sratio = float(s->sratio);
    J.invG2 = 1.0f / float(s->gspatial * s->gspatial);
    J.margin = float(s->ar);
    J.clampHull = s->ar >= 0.0;
    J.guided = guided;
    J.rw = double(sw) / cw;
    J.rh = double(sh) / ch;
    J.shiftX = -0.5;
    J.shiftY = 0.0;
    if (guided) {
        J.lcXb = sz->lcXb; J.lcXe = sz->lcXe; J.lcYb = sz->lcYb; J.lcYe = sz->lcYe;
    }
    if (e == cudaSuccess)
        e = launchSharpen(J, st);
    if (host)
        for (int p = 0; p < 3 && e == cudaSuccess; ++p) {
            const int pw = p ? cw : sw, ph = p ? ch : sh;
            e = copyPlane(out[p].data, out[p].stride, ws->stageOut[p], ws->pitch[p],
                          size_t(pw) * bps, ph, cudaMemcpyDeviceToHost, st);
        }
    if (e == cudaSuccess)
        e = cudaEventRecord(ws->done, st);
    ws->used = true;
    s->release(ws);
    if (e == cudaSuccess && host)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return cudaFail(e, "lgcr_sharpen_frame");
    return LGCR_OK;
}

} // extern "C"
