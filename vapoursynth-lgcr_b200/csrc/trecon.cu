// C ABI of TRecon (include/lgcr_b200.h): tReconCreate / tReconGetFrame /
// lgcrFree of the reference (src/plugin.cpp:723-990) on the B200 Recon path.
//
// A TRecon frame is the Recon pipeline (algo 2, lanczos taps=3, sparse off
// unless asked, mutual gate over every chroma sample) whose guided pass also
// takes the temporal taps: before it, the preparation stages convert the
// frame and its neighbours, build the neighbours' footprint maps, match
// 16x16 luma blocks against every neighbour and scale each block's
// confidence by its chroma consistency. Workspaces for those stages are
// pooled per filter.
#include "impl.h"
#include "trecon.h"

#include <algorithm>
#include <cmath>
#include <cstring>

using namespace lgcr_b200;

namespace {

bool givenInt(int v) { return v != LGCR_UNSET_INT; }
bool givenDouble(double v) { return !std::isnan(v); }

// Temporal buffers of one frame in flight: float planes of the frame and
// its neighbours, the neighbours' maps and motion fields, raw staging for
// host-memory neighbours, and the TemporalView array.
struct TReconWorkspace {
    int frames = 0;                     // capacity: 1 + neighbours
    bool host = false;
    DeviceArena arena;
    TReconPrep prep{};
    void *stage[kTReconMaxFrames][3] = {};
    size_t pitch[3] = {0, 0, 0};
    TemporalView *dViews = nullptr, *hViews = nullptr;
    cudaEvent_t done = nullptr;
    bool used = false;
    ~TReconWorkspace() {
        if (hViews) cudaFreeHost(hViews);
        if (done) cudaEventDestroy(done);
    }
};

} // namespace

struct lgcr_trecon {
    Filter *filter = nullptr;           // the Recon filter of the spatial pass
    double strength = 0.8;
    int trad = 1, tsearch = 6, numFrames = 0;
    double tsad = 0.02;
    float nw[2][129] = {};              // phase-novelty factors per axis, mv + 64
    float *dNw = nullptr;               // their device copy (first frame call)
    std::mutex mu;
    std::vector<std::unique_ptr<TReconWorkspace>> idle;
    ~lgcr_trecon() {
        delete filter;
        if (dNw) cudaFree(dNw);
    }

    const float *deviceNw() {
        std::lock_guard<std::mutex> lock(mu);
        if (!dNw) {
            float *p = nullptr;
            if (cudaMalloc(&p, sizeof(nw)) != cudaSuccess)
                return nullptr;
            if (cudaMemcpy(p, nw, sizeof(nw), cudaMemcpyHostToDevice) != cudaSuccess) {
                cudaFree(p);
                return nullptr;
            }
            dNw = p;
        }
        return dNw;
    }

    TReconWorkspace *acquire(int frames, bool host) {
        {
            std::lock_guard<std::mutex> lock(mu);
            for (size_t i = 0; i < idle.size(); ++i)
                if (idle[i]->frames >= frames && (idle[i]->host || !host)) {
                    TReconWorkspace *w = idle[i].release();
                    idle.erase(idle.begin() + i);
                    return w;
                }
        }
        const Filter &F = *filter;
        auto w = std::make_unique<TReconWorkspace>();
        w->frames = frames;
        w->host = host;
        const size_t L = size_t(F.sw) * F.sh, C = size_t(F.cw) * F.ch;
        const int bw = (F.sw + kTReconBlock - 1) / kTReconBlock;
        const int bh = (F.sh + kTReconBlock - 1) / kTReconBlock;
        const size_t B = size_t(bw) * bh;
        const int bps = F.bytesPerSample();
        size_t of[kTReconMaxFrames][3], olc[kTReconMaxFrames], omx[kTReconMaxFrames],
            omy[kTReconMaxFrames], ocf[kTReconMaxFrames], ost[kTReconMaxFrames][3];
        for (int k = 0; k < frames; ++k) {
            of[k][0] = w->arena.reserve(L * 4);
            of[k][1] = w->arena.reserve(C * 4);
            of[k][2] = w->arena.reserve(C * 4);
            olc[k] = w->arena.reserve(C * 4);
            omx[k] = w->arena.reserve(B * 2);
            omy[k] = w->arena.reserve(B * 2);
            ocf[k] = w->arena.reserve(B * 4);
            for (int p = 0; p < 3; ++p)
                ost[k][p] = (host && k > 0) ? w->arena.reserve((p ? C : L) * bps) : 0;
        }
        const size_t oViews = w->arena.reserve(sizeof(TemporalView) * kTReconMaxFrames);
        if (!w->arena.commit() ||
            cudaHostAlloc((void **)&w->hViews, sizeof(TemporalView) * kTReconMaxFrames,
                          cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&w->done, cudaEventDisableTiming) != cudaSuccess)
            return nullptr;
        w->dViews = (TemporalView *)w->arena.at(oViews);
        w->pitch[0] = size_t(F.sw) * bps;
        w->pitch[1] = w->pitch[2] = size_t(F.cw) * bps;
        for (int k = 0; k < frames; ++k) {
            for (int p = 0; p < 3; ++p) {
                w->prep.f[k][p] = (float *)w->arena.at(of[k][p]);
                if (host && k > 0)
                    w->stage[k][p] = w->arena.at(ost[k][p]);
            }
            w->prep.lc[k] = (float *)w->arena.at(olc[k]);
            w->prep.mvx[k] = (short *)w->arena.at(omx[k]);
            w->prep.mvy[k] = (short *)w->arena.at(omy[k]);
            w->prep.conf[k] = (float *)w->arena.at(ocf[k]);
        }
        w->prep.bw = bw;
        w->prep.bh = bh;
        return w.release();
    }

    void release(TReconWorkspace *w) {
        std::lock_guard<std::mutex> lock(mu);
        idle.emplace_back(w);
        if (idle.size() > 4)
            idle.erase(idle.begin());
    }
};

extern "C" {

void lgcr_trecon_params_init(lgcr_trecon_params *p) {
    if (!p)
        return;
    p->strength = p->sigma = p->sratio = p->sdb = p->gsigma = p->stretch = p->ar = NAN;
    p->ridge = p->sparse = LGCR_UNSET_INT;
    p->ms = NAN;
    p->trad = p->tsearch = LGCR_UNSET_INT;
    p->tsad = NAN;
    p->bm = LGCR_UNSET_INT;
}

int lgcr_trecon_create(const lgcr_trecon_params *params, const lgcr_format *fmt, int num_frames,
                       lgcr_trecon **out, char *err, size_t errlen) {
    auto fail = [&](const std::string &msg) {
        setError(msg);
        if (err && errlen) {
            std::strncpy(err, msg.c_str(), errlen - 1);
            err[errlen - 1] = '\0';
        }
        return LGCR_E_INVALID;
    };
    if (!fmt || !out)
        return fail("TRecon: null argument");
    lgcr_trecon_params a;
    lgcr_trecon_params_init(&a);
    if (params)
        a = *params;
    // tReconCreate src/plugin.cpp:926-966
    const bool isFloat = fmt->sample_type == LGCR_ST_FLOAT;
    if (fmt->color_family != LGCR_CF_YUV || (isFloat && fmt->bits_per_sample != 32) ||
        (!isFloat && (fmt->bits_per_sample < 8 || fmt->bits_per_sample > 16)) ||
        fmt->subsampling_w > 1 || fmt->subsampling_h > 1 || fmt->subsampling_w < 0 ||
        fmt->subsampling_h < 0)
        return fail("TRecon: planar YUV 444/422/420, 8-16 bit int or 32 bit float");
    if (fmt->width <= 0 || fmt->height <= 0 || num_frames <= 0)
        return fail("TRecon: constant dimensions and frame count required");
    const double strength = givenDouble(a.strength) ? a.strength : 0.8;
    const double sigma = givenDouble(a.sigma) ? a.sigma : 0.01;
    const double sratio = givenDouble(a.sratio) ? a.sratio : 0.15;
    const double sdb = givenDouble(a.sdb) ? a.sdb : 3.0;
    const double gsigma = givenDouble(a.gsigma) ? a.gsigma : 2.5;
    const double stretch = givenDouble(a.stretch) ? a.stretch : 1.0;
    const double ar = givenDouble(a.ar) ? a.ar : 0.0;
    const double ms = givenDouble(a.ms) ? a.ms : 1.0;
    const int trad = givenInt(a.trad) ? a.trad : 1;
    const int tsearch = givenInt(a.tsearch) ? a.tsearch : 6;
    const double tsad = givenDouble(a.tsad) ? a.tsad : 0.02;
    if (strength < 0.0 || strength > 1.0 || sigma <= 0.0 || sratio <= 0.0 || sdb <= 0.0 ||
        stretch < 0.0 || gsigma <= 0.0 || ms < 0.0 || ms > 1.0 || trad < 0 || trad > 8 ||
        tsearch < 0 || tsearch > 64 || tsad <= 0.0)
        return fail("TRecon: invalid parameter range (need 0<=strength<=1, "
                    "sigma/sratio/sdb/gsigma/tsad>0, stretch>=0, 0<=trad<=8, 0<=tsearch<=64)");
    // the spatial pass: Recon algo 2 with a lanczos3 base, sparse off unless
    // asked (src/plugin.cpp:966-977)
    lgcr_params rp;
    lgcr_params_init(&rp);
    rp.kernel = "lanczos";
    rp.taps = 3;
    rp.algo = 2;
    rp.strength = strength;
    rp.sigma = sigma;
    rp.sratio = sratio;
    rp.sdb = sdb;
    rp.gsigma = gsigma;
    rp.stretch = stretch;
    rp.ar = ar;
    rp.ms = ms;
    rp.ridge = givenInt(a.ridge) ? (a.ridge != 0) : 1;
    rp.sparse = givenInt(a.sparse) ? (a.sparse != 0) : 0;
    rp.bm = givenInt(a.bm) ? (a.bm != 0) : 0;
    std::string msg;
    Filter *f = nullptr;
    if (createFilter(&rp, fmt, &f, msg) != LGCR_OK)
        return fail("TRecon: " + msg);
    auto t = std::make_unique<lgcr_trecon>();
    t->filter = f;
    t->strength = strength;
    t->trad = trad;
    t->tsearch = tsearch;
    t->tsad = tsad;
    t->numFrames = num_frames;
    // phase-novelty factor |sin(pi * frac(mv / r))| of moving blocks
    // (src/recon.cpp:718-723), tabulated per integer motion on the host with
    // the same float arithmetic
    const float fr[2] = { float(double(f->sw) / f->cw), float(double(f->sh) / f->ch) };
    for (int axis = 0; axis < 2; ++axis)
        for (int mv = -64; mv <= 64; ++mv) {
            const float fx = float(mv) / fr[axis];
            const float px = fx - std::floor(fx);
            t->nw[axis][mv + 64] = std::fabs(std::sin(float(M_PI) * px));
        }
    *out = t.release();
    return LGCR_OK;
}

void lgcr_trecon_destroy(lgcr_trecon *t) {
    if (!t)
        return;
    cudaDeviceSynchronize();
    delete t;
}

// temporalFrameNumbers, src/plugin.cpp:729-738
int lgcr_trecon_neighbors(const lgcr_trecon *t, int n, int *frames, int cap) {
    if (!t)
        return 0;
    const int nLast = t->numFrames - 1;
    int count = 0;
    int list[2 * 8];
    for (int k = -t->trad; k <= t->trad; ++k) {
        const int fn = std::clamp(n + k, 0, nLast);
        if (fn == n || std::find(list, list + count, fn) != list + count)
            continue;
        list[count++] = fn;
    }
    for (int i = 0; i < count && i < cap && frames; ++i)
        frames[i] = list[i];
    return count;
}

int lgcr_trecon_frame(lgcr_trecon *t, const lgcr_plane cur[3], const lgcr_plane *nbrs, int count,
                      const lgcr_plane out[3], int chroma_location, int memory, void *stream) {
    if (!t || !cur || !out || count < 0 || (count > 0 && !nbrs)) {
        setError("TRecon: null argument");
        return LGCR_E_ARGUMENT;
    }
    Filter &F = *t->filter;
    const int bps = F.bytesPerSample();
    if (count > 2 * t->trad || count + 1 > kTReconMaxFrames) {
        setError("TRecon: more neighbour frames than 2 * trad");
        return LGCR_E_ARGUMENT;
    }
    auto okPlane = [&](const lgcr_plane &p, int w, int h) {
        return p.data && p.width == w && p.height == h && p.stride >= (ptrdiff_t)w * bps;
    };
    bool ok = okPlane(cur[0], F.sw, F.sh) && okPlane(cur[1], F.cw, F.ch) &&
              okPlane(cur[2], F.cw, F.ch);
    for (int p = 0; p < 3; ++p)
        ok = ok && okPlane(out[p], F.sw, F.sh);
    for (int k = 0; k < count && ok; ++k)
        ok = okPlane(nbrs[3 * k], F.sw, F.sh) && okPlane(nbrs[3 * k + 1], F.cw, F.ch) &&
             okPlane(nbrs[3 * k + 2], F.cw, F.ch);
    if (!ok) {
        setError("TRecon: plane dimensions or strides do not match the clip format");
        return LGCR_E_ARGUMENT;
    }
    if (memory != LGCR_MEM_HOST && memory != LGCR_MEM_DEVICE) {
        setError("TRecon: memory must be LGCR_MEM_HOST or LGCR_MEM_DEVICE");
        return LGCR_E_ARGUMENT;
    }
    const bool host = memory == LGCR_MEM_HOST;
    const bool temporal = t->strength > 0.0 && count > 0;
    const float *dNw = temporal ? t->deviceNw() : nullptr;
    if (temporal && !dNw) {
        setError("TRecon: device table allocation failed");
        return LGCR_E_NOMEM;
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : (host ? callingThreadStream() : nullptr);
    FrameTask task;
    task.filter = &F;
    task.p = F.sited(chroma_location);
    task.tables = F.tablesFor(task.p.shiftX, task.p.shiftY);
    if (!task.tables) {
        setError("TRecon: failed to upload geometry tables");
        return LGCR_E_NOMEM;
    }
    Workspace *ws = F.acquire(true);
    if (!ws) {
        setError("TRecon: device workspace allocation failed");
        return LGCR_E_NOMEM;
    }
    if (ws->used)
        cudaEventSynchronize(ws->done);             // its pinned job slot is rewritten
    TReconWorkspace *tw = temporal ? t->acquire(1 + count, host) : nullptr;
    if (temporal && !tw) {
        F.release(ws);
        setError("TRecon: device workspace allocation failed");
        return LGCR_E_NOMEM;
    }
    cudaError_t e = cudaSuccess;
    if (tw && tw->used)
        e = cudaEventSynchronize(tw->done);         // its pinned views are rewritten
    task.ws = ws;
    for (int p = 0; p < 3; ++p) {
        if (host) {
            if (e == cudaSuccess)
                e = copyPlane(ws->stageIn[p], ws->stageInPitch[p], cur[p].data, cur[p].stride,
                              size_t(cur[p].width) * bps, cur[p].height, cudaMemcpyHostToDevice, s);
            task.in[p] = { ws->stageIn[p], (ptrdiff_t)ws->stageInPitch[p], cur[p].width,
                           cur[p].height };
            task.out[p] = { ws->stageOut[p], (ptrdiff_t)ws->stageOutPitch[p], F.sw, F.sh };
        } else {
            task.in[p] = cur[p];
            task.out[p] = out[p];
        }
    }
    FrameJob &J = *ws->hJob;
    buildJob(task, J);
    J.lumaNormalize = F.isFloat() ? 1 : 0;
    J.gateDense = 1;
    J.shiftXd = task.p.shiftX;
    J.shiftYd = task.p.shiftY;
    if (temporal && e == cudaSuccess) {
        TReconPrep &P = tw->prep;
        P.sw = F.sw; P.sh = F.sh; P.cw = F.cw; P.ch = F.ch;
        P.kind = J.inKind;
        P.frames = 1 + count;
        P.yScale = J.yScale;
        P.cOffset = J.cOffset;
        P.search = t->tsearch;
        P.tsad = float(t->tsad);
        P.rw = J.rw;
        P.rh = J.rh;
        P.lcXb = J.lcXb; P.lcXe = J.lcXe; P.lcYb = J.lcYb; P.lcYe = J.lcYe;
        for (int p = 0; p < 3; ++p) {
            P.in[0][p] = task.in[p].data;
            P.inPitch[0][p] = task.in[p].stride;
        }
        for (int k = 1; k <= count && e == cudaSuccess; ++k)
            for (int p = 0; p < 3 && e == cudaSuccess; ++p) {
                const lgcr_plane &np = nbrs[3 * (k - 1) + p];
                if (host) {
                    e = copyPlane(tw->stage[k][p], tw->pitch[p], np.data, np.stride,
                                  size_t(np.width) * bps, np.height, cudaMemcpyHostToDevice, s);
                    P.in[k][p] = tw->stage[k][p];
                    P.inPitch[k][p] = (long long)tw->pitch[p];
                } else {
                    P.in[k][p] = np.data;
                    P.inPitch[k][p] = np.stride;
                }
            }
        for (int k = 1; k <= count; ++k)
            tw->hViews[k - 1] = { P.f[k][1], P.f[k][2], P.lc[k], P.mvx[k], P.mvy[k], P.conf[k],
                                  P.bw, P.bh };
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(tw->dViews, tw->hViews, sizeof(TemporalView) * count,
                                cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && launchTReconPrep(P, s) < 0)
            e = cudaGetLastError();
        J.tnb = tw->dViews;
        J.tnbCount = count;
        J.tnwX = dNw;
        J.tnwY = dNw + 129;
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ws->dJob, ws->hJob, sizeof(FrameJob), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        std::vector<FrameJob> jobs(1, J);
        StagePlan plan;
        planStages(jobs, plan);
        if (launchStages(jobs, plan, ws->dJob, singleFramePrefix(), s) < 0)
            e = cudaGetLastError();
    }
    if (host)
        for (int p = 0; p < 3 && e == cudaSuccess; ++p)
            e = copyPlane(out[p].data, out[p].stride, ws->stageOut[p], ws->stageOutPitch[p],
                          size_t(F.sw) * bps, F.sh, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaEventRecord(ws->done, s);
    ws->used = true;
    F.release(ws);
    if (tw) {
        if (e == cudaSuccess)
            e = cudaEventRecord(tw->done, s);
        tw->used = true;
        t->release(tw);
    }
    if (e == cudaSuccess && host)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return cudaFail(e, "lgcr_trecon_frame");
    return LGCR_OK;
}

} // extern "C"
