// C ABI of the B200 Recon path (include/lgcr_b200.h): the per-frame drop-in
// for lgcrGetFrame plus create/destroy/format queries.
#include "impl.h"

#include <cmath>
#include <cstring>

using namespace lgcr_b200;

namespace lgcr_b200 {
const char *lastError();
}

namespace lgcr_b200 {

// Stage prefix table of a single-frame launch (every stage starts at block
// 0): zeros, shared by all single-frame calls.
const int *singleFramePrefix() {
    static int *buf = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        if (cudaMalloc(&buf, 4096 * sizeof(int)) == cudaSuccess)
            cudaMemset(buf, 0, 4096 * sizeof(int));
    });
    return buf;
}

// The calling host thread's own non-blocking stream (host-memory calls
// without a caller stream).
cudaStream_t callingThreadStream() {
    thread_local cudaStream_t s = nullptr;
    if (!s)
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    return s;
}

} // namespace lgcr_b200

namespace {

// Completion event of the calling thread's frames (blocking sync), or null.
cudaEvent_t threadDoneEvent() {
    thread_local cudaEvent_t ev = nullptr;
    if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming | cudaEventBlockingSync) != cudaSuccess)
        ev = nullptr;
    return ev;
}

// Page-locked (or otherwise device-accessible) host memory: the DMA engine
// reads or writes it directly.
bool pinnedHost(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}

// Host rows between a strided caller plane and a packed staging buffer.
void copyRows(void *dst, size_t dpitch, const void *src, size_t spitch, size_t rowBytes,
              size_t rows) {
    for (size_t r = 0; r < rows; ++r)
        std::memcpy(static_cast<char *>(dst) + r * dpitch,
                    static_cast<const char *>(src) + r * spitch, rowBytes);
}

bool checkPlane(const lgcr_plane &p, int w, int h, int bps, bool allowNull) {
    if (!p.data)
        return allowNull;
    return p.width == w && p.height == h && p.stride >= (ptrdiff_t)w * bps;
}

} // namespace

extern "C" {

void lgcr_params_init(lgcr_params *p) {
    if (!p)
        return;
    p->width = p->height = LGCR_UNSET_INT;
    p->kernel = nullptr;
    p->taps = LGCR_UNSET_INT;
    p->algo = LGCR_UNSET_INT;
    p->b = p->c = NAN;
    p->strength = p->sigma = p->sratio = p->sdb = p->stretch = p->gsigma = p->rescue = NAN;
    p->ridge = p->cedge = LGCR_UNSET_INT;
    p->ar = p->reg = NAN;
    p->loc = nullptr;
    p->sparse = LGCR_UNSET_INT;
    p->bp = p->ms = p->qgate = NAN;
    p->bm = LGCR_UNSET_INT;
}

const char *lgcr_last_error(void) { return lastError(); }

int lgcr_recon_create(const lgcr_params *params, const lgcr_format *fmt, lgcr_recon **out,
                      char *err, size_t errlen) {
    std::string msg;
    Filter *f = nullptr;
    const int status = createFilter(params, fmt, &f, msg);
    if (status != LGCR_OK) {
        setError(msg);
        if (err && errlen) {
            std::strncpy(err, msg.c_str(), errlen - 1);
            err[errlen - 1] = '\0';
        }
        return status;
    }
    *out = new lgcr_recon{f};
    return LGCR_OK;
}

void lgcr_recon_destroy(lgcr_recon *h) {
    if (!h)
        return;
    cudaDeviceSynchronize();
    delete h->filter;
    delete h;
}

int lgcr_recon_output_format(const lgcr_recon *h, lgcr_format *out) {
    if (!h || !out)
        return LGCR_E_ARGUMENT;
    *out = h->filter->fmt;
    out->subsampling_w = out->subsampling_h = 0;
    out->width = h->filter->p.outW;
    out->height = h->filter->p.outH;
    return LGCR_OK;
}

int lgcr_recon_frame(lgcr_recon *h, const lgcr_plane in[3], const lgcr_plane out[3],
                     int chroma_location, int memory, void *stream, lgcr_frame_stats *stats) {
    if (!h || !in || !out) {
        setError("LGCR: null argument");
        return LGCR_E_ARGUMENT;
    }
    Filter &F = *h->filter;
    const int bps = F.bytesPerSample();
    const bool sameSize = F.p.outW == F.sw && F.p.outH == F.sh;
    if (!checkPlane(in[0], F.sw, F.sh, bps, false) || !checkPlane(in[1], F.cw, F.ch, bps, false) ||
        !checkPlane(in[2], F.cw, F.ch, bps, false) ||
        !checkPlane(out[0], F.p.outW, F.p.outH, bps, sameSize) ||
        !checkPlane(out[1], F.p.outW, F.p.outH, bps, false) ||
        !checkPlane(out[2], F.p.outW, F.p.outH, bps, false)) {
        setError("LGCR: plane dimensions or strides do not match the clip format");
        return LGCR_E_ARGUMENT;
    }
    if (memory != LGCR_MEM_HOST && memory != LGCR_MEM_DEVICE) {
        setError("LGCR: memory must be LGCR_MEM_HOST or LGCR_MEM_DEVICE");
        return LGCR_E_ARGUMENT;
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : (memory == LGCR_MEM_HOST ? callingThreadStream() : nullptr);
    FrameTask t;
    t.filter = &F;
    t.p = F.sited(chroma_location);
    t.tables = F.tablesFor(t.p.shiftX, t.p.shiftY);
    if (!t.tables) {
        setError("LGCR: failed to upload geometry tables");
        return LGCR_E_NOMEM;
    }
    Workspace *ws = F.acquire();
    if (!ws) {
        setError("LGCR: device workspace allocation failed");
        return LGCR_E_NOMEM;
    }
    // the pinned job slot is rewritten below: the previous frame that used
    // this workspace must have consumed it
    if (ws->used)
        cudaEventSynchronize(ws->done);
    t.ws = ws;
    cudaError_t e = cudaSuccess;
    bool pageableOut[3] = {false, false, false};
    if (memory == LGCR_MEM_HOST) {
        for (int i = 0; i < 3; ++i) {
            const size_t rowBytes = size_t(in[i].width) * bps, rows = in[i].height;
            if (pinnedHost(in[i].data)) {
                e = copyPlane(ws->stageIn[i], ws->stageInPitch[i], in[i].data, in[i].stride,
                              rowBytes, rows, cudaMemcpyHostToDevice, s);
            } else {
                // pageable caller memory (a VapourSynth frame): stage it in this
                // workspace's pinned buffer, then one DMA
                if (!ws->pinnedIn[i])
                    e = cudaHostAlloc(&ws->pinnedIn[i], rowBytes * rows, cudaHostAllocDefault);
                if (e == cudaSuccess) {
                    copyRows(ws->pinnedIn[i], rowBytes, in[i].data, in[i].stride, rowBytes, rows);
                    e = copyPlane(ws->stageIn[i], ws->stageInPitch[i], ws->pinnedIn[i], rowBytes,
                                  rowBytes, rows, cudaMemcpyHostToDevice, s);
                }
            }
            if (e != cudaSuccess) break;
            t.in[i] = { ws->stageIn[i], (ptrdiff_t)ws->stageInPitch[i], in[i].width, in[i].height };
            t.out[i] = { ws->stageOut[i], (ptrdiff_t)ws->stageOutPitch[i], F.p.outW, F.p.outH };
        }
        if (!out[0].data)
            t.out[0].data = nullptr;
    } else {
        for (int i = 0; i < 3; ++i) {
            t.in[i] = in[i];
            t.out[i] = out[i];
        }
    }
    if (e == cudaSuccess) {
        buildJob(t, *ws->hJob);
        e = cudaMemcpyAsync(ws->dJob, ws->hJob, sizeof(FrameJob), cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess) {
        std::vector<FrameJob> jobs(1, *ws->hJob);
        StagePlan plan;
        planStages(jobs, plan);
        if (launchStages(jobs, plan, ws->dJob, singleFramePrefix(), s) < 0)
            e = cudaGetLastError();
    }
    if (e == cudaSuccess && memory == LGCR_MEM_HOST) {
        for (int i = 0; i < 3 && e == cudaSuccess; ++i) {
            if (!out[i].data)
                continue;
            const size_t rowBytes = size_t(F.p.outW) * bps, rows = F.p.outH;
            if (pinnedHost(out[i].data)) {
                e = copyPlane(out[i].data, out[i].stride, ws->stageOut[i], ws->stageOutPitch[i],
                              rowBytes, rows, cudaMemcpyDeviceToHost, s);
                continue;
            }
            if (!ws->pinnedOut[i])
                e = cudaHostAlloc(&ws->pinnedOut[i], rowBytes * rows, cudaHostAllocDefault);
            if (e == cudaSuccess)
                e = copyPlane(ws->pinnedOut[i], rowBytes, ws->stageOut[i], ws->stageOutPitch[i],
                              rowBytes, rows, cudaMemcpyDeviceToHost, s);
            pageableOut[i] = true;
        }
    }
    unsigned long long counters[kCntCount] = {};
    if (e == cudaSuccess && stats)
        e = cudaMemcpyAsync(counters, ws->counters, sizeof(counters), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaEventRecord(ws->done, s);
    ws->used = true;
    const FrameJob J = *ws->hJob;
    const bool holdStaging = pageableOut[0] || pageableOut[1] || pageableOut[2];
    if (!holdStaging)
        F.release(ws);
    // wait on a blocking-sync event of this thread recorded after the frame's
    // last operation: the calling thread sleeps instead of spinning on a core
    if (e == cudaSuccess && (memory == LGCR_MEM_HOST || stats)) {
        const cudaEvent_t fin = threadDoneEvent();
        e = fin ? cudaEventRecord(fin, s) : cudaStreamSynchronize(s);
        if (fin && e == cudaSuccess)
            e = cudaEventSynchronize(fin);
    }
    if (holdStaging) {
        // pageable outputs leave the workspace's pinned buffers only now; the
        // workspace returns to the pool afterwards
        for (int i = 0; i < 3 && e == cudaSuccess; ++i)
            if (pageableOut[i]) {
                const size_t rowBytes = size_t(F.p.outW) * bps;
                copyRows(out[i].data, out[i].stride, ws->pinnedOut[i], rowBytes, rowBytes,
                         F.p.outH);
            }
        F.release(ws);
    }
    if (e != cudaSuccess)
        return cudaFail(e, "lgcr_recon_frame");
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->output_pixels = uint64_t(J.W) * J.H;
        if (J.sparse) {
            stats->sparse_active_pixels = counters[kCntMaskPixels];
            stats->sparse_total_pixels = uint64_t(J.sw) * J.sh;
            stats->active_output_pixels = counters[kCntActiveOutput];
            stats->active_chroma_pixels = counters[kCntActiveChroma];
            stats->sparse_active_ratio = double(counters[kCntMaskPixels]) / (double(J.sw) * J.sh);
        } else {
            stats->active_output_pixels = stats->output_pixels;
            stats->active_chroma_pixels = uint64_t(J.cw) * J.ch;
            stats->sparse_active_ratio = 1.0;
        }
    }
    return LGCR_OK;
}

int lgcr_debug_axis(const lgcr_recon *h, int axis, double shift, int *start, float *w,
                    uint8_t *am, float *pos, float *lpos, int *ci0, float *cf, int *li0,
                    float *lf, int *sup) {
    if (!h || !sup)
        return LGCR_E_ARGUMENT;
    const Filter &F = *h->filter;
    const int srcN = axis == 0 ? F.sw : F.sh;
    const int dstN = axis == 0 ? F.p.outW : F.p.outH;
    const double r = axis == 0 ? double(F.sw) / F.cw : double(F.sh) / F.ch;
    const ChromaAxis a = buildChromaAxis(srcN, dstN, r, shift, F.p.k);
    *sup = a.sup;
    for (int i = 0; i < a.n; ++i) {
        if (start) start[i] = a.start[i];
        if (pos) pos[i] = a.pos[i];
        if (lpos) lpos[i] = a.lpos[i];
        if (ci0) ci0[i] = a.chromaBilin.i0[i];
        if (cf) cf[i] = a.chromaBilin.f[i];
        if (li0) li0[i] = a.lumaBilin.i0[i];
        if (lf) lf[i] = a.lumaBilin.f[i];
        for (int j = 0; j < a.sup; ++j) {
            if (w) w[size_t(i) * a.sup + j] = a.w[size_t(i) * a.sup + j];
            if (am) am[size_t(i) * a.sup + j] = a.am[size_t(i) * a.sup + j];
        }
    }
    return LGCR_OK;
}

} // extern "C"
