// Host runtime of the B200 Recon path: filters, resident tables, device
// workspaces and the stage scheduler shared by the per-frame, batched and
// serving forms.
#pragma once

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/lgcr_b200.h"
#include "geometry.h"
#include "recon.cuh"

namespace lgcr_b200 {

// Resolved Recon arguments (the reference's LGCRData, src/lgcr.h:123-164).
struct FilterParams {
    int outW = 0, outH = 0;
    KernelSpec k;
    int taps = 6;
    double strength = 0.8, sigma = 0.01, sratio = 0.15, sdb = 3.0, reg = 0.005;
    double stretch = 1.0, gsigma = 2.5, rescue = 1.0;
    int algo = 2;
    bool ridge = true, cedge = false;
    double ms = 1.0, qgate = 1.0;
    bool sparse = true, locSet = false, bm = false;
    double bp = 0.0, arMargin = 0.0;
    double shiftX = -0.5, shiftY = 0.0;
};

// A device allocation carved into 256-byte aligned pieces.
class DeviceArena {
public:
    DeviceArena() = default;
    ~DeviceArena();
    DeviceArena(const DeviceArena &) = delete;
    DeviceArena &operator=(const DeviceArena &) = delete;
    // two-phase use: reserve() sizes, commit() allocates, then take() again
    size_t reserve(size_t bytes) { const size_t o = size_; size_ += (bytes + 255) & ~size_t(255); return o; }
    bool commit();
    void *at(size_t offset) const { return static_cast<char *>(base_) + offset; }
    size_t size() const { return size_; }
private:
    void *base_ = nullptr;
    size_t size_ = 0;
};

// Geometry tables of one (filter, chroma siting), resident in HBM.
struct DeviceTables {
    double shiftX = 0, shiftY = 0;
    DeviceArena arena;
    AxisView ax{}, ay{};
    RadialView rad{};
    WeightView lumaH{}, lumaV{};
    const int *lcXb = nullptr, *lcXe = nullptr, *lcYb = nullptr, *lcYe = nullptr;
    // algo 6
    WeightView ycH1{}, ycV1{}, ycH2{}, ycV2{};
    AxisView sax{}, say{};
    RadialView srad{};
    int nyqX = 0, nyqY = 0;
    // algo 4
    const int *lsX = nullptr, *lsY = nullptr;
    const float *lsXf = nullptr, *lsYf = nullptr;
    // bm
    const int *bmStartsX = nullptr, *bmStartsY = nullptr;
    int bmAnchorsX = 0, bmAnchorsY = 0;
    int axSup = 0, aySup = 0;
    int plainMaxRows = 0;               // most chroma rows one k_plain block reads
    int plainRows = 0;                  // output rows per k_plain block
    int detailMaxRows = 0;              // most chroma rows one k_detail_map block reads
    int detailRows = 0;                 // output rows per k_detail_map block
    int sAxSup = 0, sAySup = 0;         // source-grid axis supports (algo 6)
    int ycMaxRows = 0, ycMaxSup = 0;    // candidate tables: rows per k_yc_tiled block, widest support
};

struct Filter;

// Per-frame device workspace (planes sized for the filter's geometry).
struct Workspace {
    Filter *owner = nullptr;
    DeviceArena arena;
    FrameJob *dJob = nullptr;           // device slot for the per-frame form
    FrameJob *hJob = nullptr;           // pinned host staging of the job
    float *Yw = nullptr, *Uw = nullptr, *Vw = nullptr;
    float *jxx = nullptr, *jxy = nullptr, *jyy = nullptr, *lc = nullptr, *ms = nullptr;
    uint8_t *seed = nullptr, *mtmp = nullptr, *mask = nullptr, *cmask = nullptr;
    float *oU = nullptr, *oV = nullptr, *lumaTmp = nullptr;
    unsigned long long *counters = nullptr;
    double *uvd = nullptr;
    float *hTab = nullptr;
    float *wExt = nullptr;              // W x H float4 hull plane, then W x H float2 luma plane
    uint32_t *actList = nullptr;
    uint32_t *chromaList = nullptr;
    float *aff = nullptr, *yc1 = nullptr, *yc2 = nullptr, *ycTmp = nullptr;
    float *detail = nullptr, *detailTmp = nullptr, *detailTmp2 = nullptr, *dTab = nullptr;
    float *lgf = nullptr, *selW2 = nullptr, *selW3 = nullptr, *gU = nullptr, *gV = nullptr;
    uint8_t *roi = nullptr;
    float *bmAcc = nullptr, *bmGuide = nullptr, *bmPatch = nullptr;
    int *bmGroups = nullptr;
    void *stageIn[3] = {nullptr, nullptr, nullptr};
    void *stageOut[3] = {nullptr, nullptr, nullptr};
    size_t stageInPitch[3] = {0, 0, 0}, stageOutPitch[3] = {0, 0, 0};
    cudaEvent_t done = nullptr;
    bool used = false;
    bool hostStaging = false;           // has the host-buffer staging planes
    // pinned host copies of the planes for callers whose buffers are pageable
    // (allocated on first use): the DMA then runs from/to page-locked memory
    // and concurrent frames do not share the driver's staging buffer
    void *pinnedIn[3] = {nullptr, nullptr, nullptr};
    void *pinnedOut[3] = {nullptr, nullptr, nullptr};
    ~Workspace();
};

struct FrameTask {
    Filter *filter = nullptr;
    Workspace *ws = nullptr;
    const DeviceTables *tables = nullptr;
    FilterParams p;                     // with the frame's siting applied
    lgcr_plane in[3], out[3];           // device planes
};

struct Filter {
    FilterParams p;
    lgcr_format fmt{};
    int sw = 0, sh = 0, cw = 0, ch = 0;
    float *dLut = nullptr;
    std::mutex mu;
    std::vector<std::unique_ptr<DeviceTables>> tables;
    std::vector<std::unique_ptr<Workspace>> idle, idleBatch;   // per-frame / batched forms
    std::atomic<int> live{0}, liveBatch{0};
    ~Filter();

    const DeviceTables *tablesFor(double shiftX, double shiftY);
    // A workspace from the filter's pool (per-frame form: with host staging;
    // batched/serving forms: without). The caller must order its work after
    // the workspace's previous frame (event `done`) when `used` is set.
    Workspace *acquire(bool hostStaging = true);
    void release(Workspace *ws);
    std::unique_ptr<Workspace> makeWorkspace(bool hostStaging);
    size_t workspaceBytes();
    FilterParams sited(int chromaLocation) const;
    bool isFloat() const { return fmt.sample_type == LGCR_ST_FLOAT; }
    int bytesPerSample() const { return isFloat() ? 4 : (fmt.bits_per_sample > 8 ? 2 : 1); }
    bool directOutput(const FilterParams &q) const;
    bool needsBackProjection(const FilterParams &q) const;
};

// Creates a Filter from Recon arguments; mirrors lgcrCreate's validation.
int createFilter(const lgcr_params *params, const lgcr_format *fmt, Filter **out,
                 std::string &err);

// Scalar geometry of a table set that every builder must fill the same way:
// the chroma axes' supports (they decide buildJob's unclamped-tap and fast
// reciprocal flags) and the k_plain block height.
void setAxisGeometry(DeviceTables &t, const ChromaAxis &ax, const ChromaAxis &ay, int outH,
                     int ch);

// Fill the device FrameJob of one task.
void buildJob(const FrameTask &t, FrameJob &job);

// Stage scheduler: launches every stage once over all jobs. `dJobs` is the
// device copy of `jobs`; `dPrefix` receives the stage prefix tables (space
// for stageCount * (n + 1) ints) and is written from `hPrefix` (pinned,
// same size) by one copy. Returns the number of kernel launches, or -1.
// Launch settings a plan is made and launched with: block shapes of the
// tunable per-pixel stages and the persistent guided kernel's variant. A
// plan keeps its own copy, so its tile counts and block shapes always agree
// even when the settings change while it runs.
constexpr int kMaxStages = 64;
struct LaunchConfig {
    int shapeX[kMaxStages], shapeY[kMaxStages];
    int guidedVariant;
};
// The process-wide settings (lgcr_autotune, LGCR_GUIDED_VARIANT) and a
// counter that changes whenever they do.
LaunchConfig processLaunchConfig();
int processConfigVersion();

struct StagePlan {
    std::vector<int> prefix;            // stageCount * (n+1)
    std::vector<int> totals;            // blocks per stage
    int maxDil = 0;
    int nyqPasses = 0;
    LaunchConfig cfg;
};
int stageCount();
// cfg == nullptr: the process-wide settings at the time of the call
void planStages(const std::vector<FrameJob> &jobs, StagePlan &plan,
                const LaunchConfig *cfg = nullptr);
int launchStages(const std::vector<FrameJob> &jobs, const StagePlan &plan,
                 const FrameJob *dJobs, const int *dPrefix, cudaStream_t stream);

const char *stageName(int stage);
bool stageTunable(int stage);
void stageShape(int stage, int &bx, int &by);
void setStageShape(int stage, int bx, int by);
int guidedVariant();
void setGuidedVariant(int variant);
const char *setError(const std::string &msg);

// Plane copy between host and device: one linear copy when both sides are
// packed (pitch == row bytes), else a 2D copy.
inline cudaError_t copyPlane(void *dst, size_t dpitch, const void *src, size_t spitch,
                             size_t rowBytes, size_t rows, cudaMemcpyKind kind, cudaStream_t s) {
    if (dpitch == rowBytes && spitch == rowBytes)
        return cudaMemcpyAsync(dst, src, rowBytes * rows, kind, s);
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, rowBytes, rows, kind, s);
}
int cudaFail(cudaError_t e, const char *where);

// Zero stage prefix table for single-frame launches (device memory).
const int *singleFramePrefix();
// The calling host thread's own non-blocking stream.
cudaStream_t callingThreadStream();

} // namespace lgcr_b200

// Handle type of the C ABI.
struct lgcr_recon {
    lgcr_b200::Filter *filter;
};
