// lgcr_recon_frame_static: the per-frame Recon (algo 2, or any algo at
// strength 0) for callers that must not allocate device memory.
//
// Who needs it: hosts that own all device memory through their own pool and
// forbid libraries from calling cudaMalloc, and callers on latency-critical
// paths where cudaMalloc/cudaFree would implicitly synchronize the device.
// The regular entry point allocates a workspace and resident tables on first
// use; this one allocates nothing. Its scratch -- converted source planes,
// structure tensor, trust masks, chroma workset, counters, geometry tables
// and the frame descriptor -- lives in one file-scope device array of
// kStaticScratchBytes (64 MiB), which every GPU that loads the library holds
// until the process exits. Frames whose scratch exceeds it are rejected.
//
// The first call on each device resolves the array's device address with
// cudaGetSymbolAddress (with that device current); make that first call
// before any stream capture. Every call shares the one array and it keeps
// the previous call's contents, so everything that must start at zero is
// cleared on the stream by the call itself; calls whose work overlaps on the
// GPU (different streams, or the same device from several threads without
// ordering) race on the array and must be serialized by the caller.
#include "impl.h"
#include "kernels.cuh"

#include <cmath>
#include <cstring>
#include <mutex>

using namespace lgcr_b200;

namespace {

constexpr size_t kStaticScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_staticScratch[kStaticScratchBytes];

std::mutex gAddrMu;
unsigned char *gAddr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set up once).
cudaError_t scratchAddress(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (dev < 0 || dev >= kMaxDevices)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(gAddrMu);
    if (!gAddr[dev]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_staticScratch);
        if (e != cudaSuccess)
            return e;
        gAddr[dev] = static_cast<unsigned char *>(ptr);
    }
    *out = gAddr[dev];
    return cudaSuccess;
}

// Host image of the region: arrays appended at 256-byte aligned offsets.
struct Image {
    std::vector<uint8_t> bytes;
    template <class T> size_t add(const std::vector<T> &v) {
        const size_t off = (bytes.size() + 255) & ~size_t(255);
        bytes.resize(off + v.size() * sizeof(T));
        if (!v.empty())
            std::memcpy(bytes.data() + off, v.data(), v.size() * sizeof(T));
        return off;
    }
};

} // namespace

extern "C" int lgcr_recon_frame_static(lgcr_recon *h, const lgcr_plane in[3],
                                       const lgcr_plane out[3], int chroma_location,
                                       void *stream) {
    if (!h || !in || !out) {
        setError("LGCR: null argument");
        return LGCR_E_ARGUMENT;
    }
    // the uploads read host memory that is gone when the call returns: a
    // captured copy node would read it again at every replay
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing((cudaStream_t)stream, &capturing) == cudaSuccess &&
        capturing != cudaStreamCaptureStatusNone) {
        setError("LGCR: lgcr_recon_frame_static cannot be captured into a CUDA graph "
                 "(its table uploads read host memory owned by the call)");
        return LGCR_E_ARGUMENT;
    }
    Filter &F = *h->filter;
    const FilterParams q = F.sited(chroma_location);
    if (q.bm || F.needsBackProjection(q) || (q.strength > 0.0 && q.algo != 2)) {
        setError("LGCR: lgcr_recon_frame_static runs algo=2 (or strength=0) without bm/bp");
        return LGCR_E_ARGUMENT;
    }
    const int bps = F.bytesPerSample();
    const bool sameSize = q.outW == F.sw && q.outH == F.sh;
    auto okPlane = [&](const lgcr_plane &p, int w, int hgt, bool allowNull) {
        if (!p.data) return allowNull;
        return p.width == w && p.height == hgt && p.stride >= (ptrdiff_t)w * bps;
    };
    if (!okPlane(in[0], F.sw, F.sh, false) || !okPlane(in[1], F.cw, F.ch, false) ||
        !okPlane(in[2], F.cw, F.ch, false) || !okPlane(out[0], q.outW, q.outH, sameSize) ||
        !okPlane(out[1], q.outW, q.outH, false) || !okPlane(out[2], q.outW, q.outH, false)) {
        setError("LGCR: plane dimensions or strides do not match the clip format");
        return LGCR_E_ARGUMENT;
    }
    unsigned char *base = nullptr;
    cudaError_t e = scratchAddress(&base);
    if (e != cudaSuccess)
        return cudaFail(e, "lgcr_recon_frame_static (scratch address)");

    // geometry tables (host-built, uploaded into the scratch array)
    const double rw = double(F.sw) / F.cw, rh = double(F.sh) / F.ch;
    const ChromaAxis ax = buildChromaAxis(F.sw, q.outW, rw, q.shiftX, q.k);
    const ChromaAxis ay = buildChromaAxis(F.sh, q.outH, rh, q.shiftY, q.k);
    Image img;
    struct AxisOff { size_t s, w, wd, am, ws, wa, pos, lpos, ci, cf, li, lf, kmx, kss; } oa[2];
    const ChromaAxis *axes[2] = { &ax, &ay };
    for (int i = 0; i < 2; ++i) {
        const ChromaAxis &a = *axes[i];
        const std::vector<double> wd(a.w.begin(), a.w.end());
        std::vector<float> kmx, kss;
        rescueFactors(a, kmx, kss);
        oa[i] = { img.add(a.start), img.add(a.w), img.add(wd), img.add(a.am), img.add(a.weightSum),
                  img.add(a.absoluteWeightSum), img.add(a.pos), img.add(a.lpos),
                  img.add(a.chromaBilin.i0), img.add(a.chromaBilin.f),
                  img.add(a.lumaBilin.i0), img.add(a.lumaBilin.f), img.add(kmx), img.add(kss) };
    }
    RadialTable rad;
    size_t orx = 0, ory = 0, orw = 0;
    if (q.k.radial) {
        rad = buildRadialTable(q.k, ax, ay, F.cw, F.ch);
        if (rad.valid) {
            orx = img.add(rad.xPhase); ory = img.add(rad.yPhase); orw = img.add(rad.weights);
        }
    }
    WeightTable lh, lv;
    size_t olhs = 0, olhw = 0, olvs = 0, olvw = 0;
    if (!sameSize && !q.k.radial) {
        lh = buildWeights(F.sw, q.outW, q.k, 0.0);
        lv = buildWeights(F.sh, q.outH, q.k, 0.0);
        olhs = img.add(lh.start); olhw = img.add(lh.w);
        olvs = img.add(lv.start); olvw = img.add(lv.w);
    }
    std::vector<int> xb, xe, yb, ye;
    lcExtents(F.sw, F.cw, rw, q.shiftX, xb, xe);
    lcExtents(F.sh, F.ch, rh, q.shiftY, yb, ye);
    const size_t oxb = img.add(xb), oxe = img.add(xe), oyb = img.add(yb), oye = img.add(ye);
    const size_t tableBytes = (img.bytes.size() + 255) & ~size_t(255);

    // workspace planes after the tables
    size_t cursor = tableBytes;
    auto take = [&](size_t bytes) { const size_t o = cursor; cursor += (bytes + 255) & ~size_t(255); return o; };
    const size_t L = size_t(F.sw) * F.sh, C = size_t(F.cw) * F.ch;
    const bool guided = q.strength > 0.0;
    const bool sparse = guided && q.sparse;
    const size_t oJob = take(sizeof(FrameJob)), oPrefix = take(4096 * sizeof(int));
    const size_t oCnt = take(kCntCount * sizeof(unsigned long long));
    const size_t oY = take(L * 4), oU = take(C * 4), oV = take(C * 4);
    const size_t oJxx = guided ? take(L * 4) : 0, oJxy = guided ? take(L * 4) : 0;
    const size_t oJyy = guided ? take(L * 4) : 0, oLc = guided ? take(C * 4) : 0;
    const size_t oMs = (guided && q.ms > 0.0) ? take(C * 4) : 0;
    const size_t maskBytes = size_t((F.sw + 31) / 32) * 4 * F.sh;
    const size_t oSeed = sparse ? take(L) : 0, oMtmp = sparse ? take(maskBytes) : 0;
    const size_t oMask = sparse ? take(maskBytes) : 0, oCmask = sparse ? take(C) : 0;
    const size_t oLumaTmp = (!sameSize && !q.k.radial) ? take(size_t(q.outW) * F.sh * 4) : 0;
    const size_t oUvd = take(C * 16);
    const size_t oList = guided ? take(size_t(q.outW) * q.outH * 4) : 0;
    if (cursor > kStaticScratchBytes) {
        char msg[200];
        std::snprintf(msg, sizeof(msg),
                      "LGCR: frame needs %zu bytes of scratch; lgcr_recon_frame_static holds %zu",
                      cursor, kStaticScratchBytes);
        setError(msg);
        return LGCR_E_ARGUMENT;
    }

    DeviceTables T;
    auto axisView = [&](const AxisOff &o, const ChromaAxis &a) {
        AxisView v;
        v.n = a.n; v.sup = a.sup;
        v.start = (const int *)(base + o.s); v.w = (const float *)(base + o.w);
        v.wd = (const double *)(base + o.wd);
        v.am = (const uint8_t *)(base + o.am); v.wsum = (const float *)(base + o.ws);
        v.wabs = (const float *)(base + o.wa); v.pos = (const float *)(base + o.pos);
        v.lpos = (const float *)(base + o.lpos); v.cbI0 = (const int *)(base + o.ci);
        v.cbF = (const float *)(base + o.cf); v.lbI0 = (const int *)(base + o.li);
        v.lbF = (const float *)(base + o.lf);
        v.kmx = (const float *)(base + o.kmx);
        v.kss = (const float *)(base + o.kss);
        v.amBits = nullptr;      // activity read from the bytes
        return v;
    };
    T.ax = axisView(oa[0], ax);
    T.ay = axisView(oa[1], ay);
    setAxisGeometry(T, ax, ay, q.outH, F.ch);
    if (q.k.radial) {
        T.rad.valid = rad.valid;
        T.rad.supX = rad.supportX; T.rad.supY = rad.supportY; T.rad.phasesX = rad.phaseCountX;
        if (rad.valid) {
            T.rad.xPhase = (const uint16_t *)(base + orx);
            T.rad.yPhase = (const uint16_t *)(base + ory);
            T.rad.weights = (const float *)(base + orw);
        }
    }
    if (!sameSize && !q.k.radial) {
        T.lumaH = { lh.n, lh.sup, (const int *)(base + olhs), (const float *)(base + olhw) };
        T.lumaV = { lv.n, lv.sup, (const int *)(base + olvs), (const float *)(base + olvw) };
    }
    T.lcXb = (const int *)(base + oxb); T.lcXe = (const int *)(base + oxe);
    T.lcYb = (const int *)(base + oyb); T.lcYe = (const int *)(base + oye);

    Workspace ws;
    auto fp = [&](size_t o) { return (float *)(base + o); };
    auto bp = [&](size_t o) { return (uint8_t *)(base + o); };
    ws.dJob = (FrameJob *)(base + oJob);
    ws.Yw = fp(oY); ws.Uw = fp(oU); ws.Vw = fp(oV);
    ws.jxx = guided ? fp(oJxx) : nullptr; ws.jxy = guided ? fp(oJxy) : nullptr;
    ws.jyy = guided ? fp(oJyy) : nullptr; ws.lc = guided ? fp(oLc) : nullptr;
    ws.ms = oMs ? fp(oMs) : nullptr;
    ws.seed = sparse ? bp(oSeed) : nullptr; ws.mtmp = sparse ? bp(oMtmp) : nullptr;
    ws.mask = sparse ? bp(oMask) : nullptr; ws.cmask = sparse ? bp(oCmask) : nullptr;
    ws.lumaTmp = oLumaTmp ? fp(oLumaTmp) : nullptr;
    ws.counters = (unsigned long long *)(base + oCnt);
    ws.uvd = (double *)(base + oUvd);
    ws.actList = guided ? (uint32_t *)(base + oList) : nullptr;
    ws.hTab = nullptr;      // plain and guided windows are read directly

    FrameTask t;
    t.filter = &F;
    t.ws = &ws;
    t.tables = &T;
    t.p = q;
    for (int i = 0; i < 3; ++i) {
        t.in[i] = in[i];
        t.out[i] = out[i];
    }
    FrameJob job;
    buildJob(t, job);
    cudaStream_t s = (cudaStream_t)stream;
    e = cudaMemcpyAsync(base, img.bytes.data(), img.bytes.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(base + oPrefix, 0, 4096 * sizeof(int), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ws.dJob, &job, sizeof(FrameJob), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess)
        return cudaFail(e, "lgcr_recon_frame_static (upload)");
    std::vector<FrameJob> jobs(1, job);
    StagePlan plan;
    planStages(jobs, plan);
    if (launchStages(jobs, plan, ws.dJob, (const int *)(base + oPrefix), s) < 0)
        return cudaFail(cudaGetLastError(), "lgcr_recon_frame_static (launch)");
    ws.dJob = nullptr;
    return LGCR_OK;
}
