// Batched form: many frames (any mix of filters, sizes, subsamplings and
// depths) per launch of each stage. The launch sequence of a batch layout is
// captured once into a CUDA graph and replayed; per-frame descriptors and
// stage prefix tables are refreshed by copy nodes that read pinned host
// buffers, so new frames (new plane pointers) replay the same graph. Runs
// rotate over a few descriptor slots (each with its graph), so a call waits
// only for the run that used its slot several calls earlier, not for the
// previous one.
#include "impl.h"
#include "kernels.cuh"

#include <cstdlib>
#include <cstring>
#include <string>

using namespace lgcr_b200;

struct StageEvent {
    int stage;
    cudaEvent_t start, stop;
};

// Descriptor buffers of one in-flight run: pinned host copies the run's
// copy nodes read, their device targets, and the event that marks them read.
// A batch cycles through kDescriptorSlots of them, so the host prepares the
// next run while the previous one executes; each slot keeps its own graph.
struct DescriptorSlot {
    FrameJob *dJobs = nullptr, *hJobs = nullptr;
    int *dPrefix = nullptr, *hPrefix = nullptr;
    cudaEvent_t done = nullptr;
    bool pending = false;
    cudaGraphExec_t exec = nullptr;     // graph of the cached layout on this slot
    std::string signature;
    int launches = 0;
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (dJobs) cudaFree(dJobs);
        if (hJobs) cudaFreeHost(hJobs);
        if (dPrefix) cudaFree(dPrefix);
        if (hPrefix) cudaFreeHost(hPrefix);
        exec = nullptr; dJobs = nullptr; hJobs = nullptr; dPrefix = nullptr; hPrefix = nullptr;
        signature.clear();
    }
};

constexpr int kDescriptorSlots = 3;

struct lgcr_batch {
    int capacity = 0;
    size_t prefixCapacity = 0;
    DescriptorSlot slots[kDescriptorSlots];
    int next = 0;                       // slot of the next run
    int lastLaunches = 0;
    // profiling
    bool profiling = false;
    std::vector<StageEvent> events;
    std::vector<cudaEvent_t> eventPool;
    std::vector<double> stageMs;
    std::vector<int> stageLaunches;
    // this batch's own launch settings (lgcr_batch_autotune); until tuned,
    // every run plans with the process-wide settings
    bool ownConfig = false;
    LaunchConfig cfg{};
    int groupMode = -2;                 // -2: process default (see batchGroupFrames)
    int cfgVersion = 0;                 // part of the graph signature
    ~lgcr_batch() {
        for (auto &sl : slots) {
            sl.release();
            if (sl.done) cudaEventDestroy(sl.done);
        }
        for (auto &e : events) { cudaEventDestroy(e.start); cudaEventDestroy(e.stop); }
        for (auto e : eventPool) cudaEventDestroy(e);
    }
};

namespace {

cudaEvent_t poolEvent(lgcr_batch *b) {
    if (!b->eventPool.empty()) {
        cudaEvent_t e = b->eventPool.back();
        b->eventPool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

int ensureCapacity(lgcr_batch *b, int count) {
    if (count <= b->capacity && size_t(stageCount()) * (2 * count) <= b->prefixCapacity)
        return LGCR_OK;
    for (auto &sl : b->slots) {
        if (sl.pending)
            cudaEventSynchronize(sl.done);
        sl.pending = false;
        sl.release();
    }
    const int cap = std::max(count, 8);
    // room for one prefix table per frame group (at most one group per frame)
    b->prefixCapacity = size_t(stageCount()) * (2 * cap);
    for (auto &sl : b->slots) {
        if (cudaMalloc(&sl.dJobs, sizeof(FrameJob) * cap) != cudaSuccess ||
            cudaHostAlloc((void **)&sl.hJobs, sizeof(FrameJob) * cap, cudaHostAllocDefault) != cudaSuccess ||
            cudaMalloc(&sl.dPrefix, b->prefixCapacity * sizeof(int)) != cudaSuccess ||
            cudaHostAlloc((void **)&sl.hPrefix, b->prefixCapacity * sizeof(int), cudaHostAllocDefault) !=
                cudaSuccess) {
            for (auto &other : b->slots)
                other.release();
            b->capacity = 0;
            b->prefixCapacity = 0;
            setError("LGCR: batch descriptor allocation failed");
            return LGCR_E_NOMEM;
        }
    }
    b->capacity = cap;
    return LGCR_OK;
}

// Frame groups of the stage sequence. Each group runs every stage before the
// next group starts, so a group's intermediate planes can still be in L2
// when its later stages read them; one group gives the fewest launches and
// the shortest tails. Measured on one B200: frames that upscale (output at
// least twice the source luma: 1080p -> 4K jinc) run their long guided pass
// 14 % faster as groups of their own (their 1080p-sized inputs stay in L2),
// while same-size frames are fastest as one group. By default every
// upscaling frame is its own group and the frames between them form one;
// LGCR_BATCH_GROUP=n (n >= 1) groups every n frames instead, 0 makes the
// whole batch one group.
int batchGroupFrames() {
    static const int g = [] {
        const char *e = std::getenv("LGCR_BATCH_GROUP");
        return e ? std::max(0, std::atoi(e)) : -1;
    }();
    return g;
}

// The batch's frame groups and their stage plans; the plans' prefix tables
// lie one after another in the slot's prefix buffer (offsets in ints).
struct GroupedPlan {
    std::vector<int> start;             // groups + 1 frame indices
    std::vector<StagePlan> plans;
    std::vector<size_t> offset;         // groups + 1
};

// groupMode: -1 upscaling frames alone, 0 one group, n >= 1 every n frames
void planGroups(const std::vector<FrameJob> &jobs, GroupedPlan &gp, int groupMode,
                const LaunchConfig *cfg) {
    const int n = int(jobs.size());
    const int g = groupMode;
    gp.start.clear();
    gp.plans.clear();
    gp.offset.assign(1, 0);
    if (g >= 0) {
        for (int f = 0; f < n; f += (g > 0 ? g : n))
            gp.start.push_back(f);
    } else {
        auto upscale = [&](int f) {
            return (long long)jobs[f].W * jobs[f].H >= 2LL * jobs[f].sw * jobs[f].sh;
        };
        for (int f = 0; f < n; ++f)
            if (f == 0 || upscale(f) || upscale(f - 1))
                gp.start.push_back(f);
    }
    gp.start.push_back(n);
    const int groups = int(gp.start.size()) - 1;
    gp.plans.resize(groups);
    for (int k = 0; k < groups; ++k) {
        const std::vector<FrameJob> sub(jobs.begin() + gp.start[k], jobs.begin() + gp.start[k + 1]);
        planStages(sub, gp.plans[k], cfg);
        gp.offset.push_back(gp.offset.back() + gp.plans[k].prefix.size());
    }
}

// Launch sequence, group by group; with profiling, each launched stage is
// bracketed by events.
int enqueue(lgcr_batch *b, DescriptorSlot &sl, const std::vector<FrameJob> &jobs,
            const GroupedPlan &gp, cudaStream_t s) {
    const int n = int(jobs.size());
    if (cudaMemcpyAsync(sl.dJobs, sl.hJobs, sizeof(FrameJob) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(sl.dPrefix, sl.hPrefix, gp.offset.back() * sizeof(int),
                        cudaMemcpyHostToDevice, s) != cudaSuccess)
        return -1;
    int launches = 0;
    for (size_t k = 0; k + 1 < gp.start.size(); ++k) {
        const std::vector<FrameJob> sub(jobs.begin() + gp.start[k], jobs.begin() + gp.start[k + 1]);
        const StagePlan &plan = gp.plans[k];
        const FrameJob *dJobs = sl.dJobs + gp.start[k];
        const int *dPrefix = sl.dPrefix + gp.offset[k];
        if (!b->profiling) {
            const int l = launchStages(sub, plan, dJobs, dPrefix, s);
            if (l < 0)
                return -1;
            launches += l;
            continue;
        }
        // profiled: one stage at a time so each launch gets its own events
        StagePlan single = plan;
        for (int st = 0; st < stageCount(); ++st) {
            if (plan.totals[st] == 0)
                continue;
            for (int o = 0; o < stageCount(); ++o)
                single.totals[o] = (o == st) ? plan.totals[st] : 0;
            StageEvent ev{st, poolEvent(b), poolEvent(b)};
            cudaEventRecord(ev.start, s);
            const int l = launchStages(sub, single, dJobs, dPrefix, s);
            cudaEventRecord(ev.stop, s);
            if (l < 0)
                return -1;
            launches += l;
            b->events.push_back(ev);
        }
    }
    return launches;
}

} // namespace

extern "C" {

int lgcr_batch_create(lgcr_batch **out) {
    if (!out)
        return LGCR_E_ARGUMENT;
    auto b = std::make_unique<lgcr_batch>();
    for (auto &sl : b->slots)
        if (cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess)
            return cudaFail(cudaGetLastError(), "lgcr_batch_create");
    b->stageMs.assign(stageCount(), 0.0);
    b->stageLaunches.assign(stageCount(), 0);
    *out = b.release();
    return LGCR_OK;
}

void lgcr_batch_destroy(lgcr_batch *b) {
    if (!b)
        return;
    cudaDeviceSynchronize();
    delete b;
}

int lgcr_batch_launch_count(const lgcr_batch *b) { return b ? b->lastLaunches : 0; }

int lgcr_batch_run(lgcr_batch *b, const lgcr_batch_item *items, int count, void *stream,
                   int use_graph) {
    if (!b || !items || count <= 0) {
        setError("LGCR: empty batch");
        return LGCR_E_ARGUMENT;
    }
    cudaStream_t s = (cudaStream_t)stream;
    int status = ensureCapacity(b, count);
    if (status != LGCR_OK)
        return status;
    // this run's pinned descriptors are rewritten: the run that last used the
    // slot (kDescriptorSlots runs ago) must have read them
    DescriptorSlot &sl = b->slots[b->next];
    if (sl.pending)
        cudaEventSynchronize(sl.done);
    sl.pending = false;
    // workspaces come from each frame's filter pool and go back after the
    // launch: a mixed stream keeps them resident across batches instead of
    // reallocating whenever a slot's filter changes
    std::vector<Workspace *> taken;
    taken.reserve(count);
    auto giveBack = [&]() {
        for (Workspace *ws : taken)
            ws->owner->release(ws);
        taken.clear();
    };
    std::vector<FrameJob> jobs(count);
    std::string sig = std::to_string(count);
    for (int i = 0; i < count; ++i) {
        const lgcr_batch_item &it = items[i];
        if (!it.filter) {
            giveBack();
            setError("LGCR: batch item without filter");
            return LGCR_E_ARGUMENT;
        }
        Filter *F = it.filter->filter;
        FrameTask t;
        t.filter = F;
        t.p = F->sited(it.chroma_location);
        t.tables = F->tablesFor(t.p.shiftX, t.p.shiftY);
        if (!t.tables) {
            giveBack();
            setError("LGCR: failed to upload geometry tables");
            return LGCR_E_NOMEM;
        }
        Workspace *ws = F->acquire(false);
        if (!ws) {
            giveBack();
            setError("LGCR: device workspace allocation failed");
            return LGCR_E_NOMEM;
        }
        if (ws->used && cudaStreamWaitEvent(s, ws->done, 0) != cudaSuccess) {
            F->release(ws);
            giveBack();
            return cudaFail(cudaGetLastError(), "lgcr_batch_run");
        }
        taken.push_back(ws);
        t.ws = ws;
        for (int p = 0; p < 3; ++p) {
            t.in[p] = it.in[p];
            t.out[p] = it.out[p];
        }
        buildJob(t, jobs[i]);
        char buf[96];
        std::snprintf(buf, sizeof(buf), "|%p,%g,%g,%d,%d", (void *)F, t.p.shiftX, t.p.shiftY,
                      t.out[0].data != nullptr, jobs[i].inKind);
        sig += buf;
    }
    GroupedPlan plan;
    planGroups(jobs, plan, b->groupMode >= -1 ? b->groupMode : batchGroupFrames(),
               b->ownConfig ? &b->cfg : nullptr);
    std::memcpy(sl.hJobs, jobs.data(), sizeof(FrameJob) * count);
    for (size_t k = 0; k < plan.plans.size(); ++k)
        std::memcpy(sl.hPrefix + plan.offset[k], plan.plans[k].prefix.data(),
                    plan.plans[k].prefix.size() * sizeof(int));
    sig += "|g" + std::to_string(plan.plans.size()) + "|c" +
           std::to_string(b->ownConfig ? b->cfgVersion : -1 - processConfigVersion());
    int launches = -1;
    // the legacy default stream cannot be captured: its runs launch directly
    const bool capturable = s != nullptr && s != cudaStreamLegacy;
    if (use_graph && !b->profiling && capturable) {
        if (!sl.exec || sl.signature != sig) {
            if (sl.exec) { cudaGraphExecDestroy(sl.exec); sl.exec = nullptr; }
            sl.signature.clear();
            cudaGraph_t graph = nullptr;
            if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                giveBack();
                return cudaFail(cudaGetLastError(), "graph capture");
            }
            launches = enqueue(b, sl, jobs, plan, s);
            const cudaError_t e = cudaStreamEndCapture(s, &graph);
            if (e != cudaSuccess || launches < 0) {
                if (graph) cudaGraphDestroy(graph);
                giveBack();
                return cudaFail(e != cudaSuccess ? e : cudaGetLastError(), "graph capture");
            }
            const cudaError_t ie = cudaGraphInstantiate(&sl.exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ie != cudaSuccess) {
                sl.exec = nullptr;
                giveBack();
                return cudaFail(ie, "graph instantiate");
            }
            sl.signature = sig;
            sl.launches = launches;
        }
        const cudaError_t e = cudaGraphLaunch(sl.exec, s);
        if (e != cudaSuccess) {
            giveBack();
            return cudaFail(e, "graph launch");
        }
        launches = sl.launches;
    } else {
        launches = enqueue(b, sl, jobs, plan, s);
        if (launches < 0) {
            giveBack();
            return cudaFail(cudaGetLastError(), "lgcr_batch_run");
        }
    }
    b->lastLaunches = launches;
    cudaEventRecord(sl.done, s);
    sl.pending = true;
    b->next = (b->next + 1) % kDescriptorSlots;
    for (Workspace *ws : taken) {
        cudaEventRecord(ws->done, s);
        ws->used = true;
    }
    giveBack();
    return LGCR_OK;
}

// Stage profiling: bracket every stage launch of subsequent runs with CUDA
// events (graphs are bypassed while on).
int lgcr_batch_set_profiling(lgcr_batch *b, int on) {
    if (!b)
        return LGCR_E_ARGUMENT;
    b->profiling = on != 0;
    return LGCR_OK;
}

// Accumulated device milliseconds and launch counts per stage since the
// last reset; waits for the recorded work. `ms`/`launches` have
// lgcr_stage_count() entries (either may be NULL).
int lgcr_batch_stage_times(lgcr_batch *b, double *ms, int *launches, int reset) {
    if (!b)
        return LGCR_E_ARGUMENT;
    for (auto &e : b->events) {
        cudaEventSynchronize(e.stop);
        float t = 0.0f;
        cudaEventElapsedTime(&t, e.start, e.stop);
        b->stageMs[e.stage] += t;
        b->stageLaunches[e.stage] += 1;
        b->eventPool.push_back(e.start);
        b->eventPool.push_back(e.stop);
    }
    b->events.clear();
    for (int i = 0; i < stageCount(); ++i) {
        if (ms) ms[i] = b->stageMs[i];
        if (launches) launches[i] = b->stageLaunches[i];
    }
    if (reset) {
        std::fill(b->stageMs.begin(), b->stageMs.end(), 0.0);
        std::fill(b->stageLaunches.begin(), b->stageLaunches.end(), 0);
    }
    return LGCR_OK;
}

int lgcr_stage_count(void) { return stageCount(); }

const char *lgcr_stage_name(int stage) { return stageName(stage); }

} // extern "C"

// Autotuner: for every tunable per-pixel stage present in the given items,
// time each candidate block (tile) shape with stage events and keep the
// fastest; the choice applies process-wide to later plans.
extern "C" int lgcr_autotune(const lgcr_batch_item *items, int count, void *stream,
                             char *report, size_t reportlen) {
    static const int cand[][2] = {{32, 8}, {16, 8}, {32, 4}, {64, 4}, {16, 16}, {128, 2}, {8, 8}};
    lgcr_batch *b = nullptr;
    int status = lgcr_batch_create(&b);
    if (status != LGCR_OK)
        return status;
    lgcr_batch_set_profiling(b, 1);
    std::string text;
    std::vector<double> ms(stageCount());
    for (int s = 0; s < stageCount() && status == LGCR_OK; ++s) {
        if (!stageTunable(s))
            continue;
        int bestX, bestY;
        stageShape(s, bestX, bestY);
        double best = 1e300;
        std::string line = std::string(stageName(s)) + ":";
        for (const auto &c : cand) {
            setStageShape(s, c[0], c[1]);
            status = lgcr_batch_run(b, items, count, stream, 0);
            if (status != LGCR_OK)
                break;
            lgcr_batch_stage_times(b, nullptr, nullptr, 1);
            for (int rep = 0; rep < 2 && status == LGCR_OK; ++rep)
                status = lgcr_batch_run(b, items, count, stream, 0);
            lgcr_batch_stage_times(b, ms.data(), nullptr, 1);
            if (ms[s] <= 0.0)
                break;                         // stage not used by these items
            char buf[64];
            std::snprintf(buf, sizeof(buf), " %dx%d=%.3fms", c[0], c[1], ms[s] / 2);
            line += buf;
            if (ms[s] < best) { best = ms[s]; bestX = c[0]; bestY = c[1]; }
        }
        setStageShape(s, bestX, bestY);
        if (best < 1e300) {
            char buf[48];
            std::snprintf(buf, sizeof(buf), " -> %dx%d\n", bestX, bestY);
            text += line + buf;
        }
    }
    // register budget of the persistent guided stage
    if (status == LGCR_OK) {
        int guidedStage = -1;
        for (int s = 0; s < stageCount(); ++s)
            if (std::string(stageName(s)) == "reconstructChroma")
                guidedStage = s;
        double best = 1e300;
        int bestV = guidedVariant();
        std::string line = "reconstructChroma:";
        static const char *names[3] = {"2-blocks", "3-blocks", "staged"};
        for (int v = 0; v < 3 && guidedStage >= 0 && status == LGCR_OK; ++v) {
            setGuidedVariant(v);
            status = lgcr_batch_run(b, items, count, stream, 0);
            lgcr_batch_stage_times(b, nullptr, nullptr, 1);
            for (int rep = 0; rep < 2 && status == LGCR_OK; ++rep)
                status = lgcr_batch_run(b, items, count, stream, 0);
            lgcr_batch_stage_times(b, ms.data(), nullptr, 1);
            if (ms[guidedStage] <= 0.0)
                break;
            char buf[64];
            std::snprintf(buf, sizeof(buf), " %s=%.3fms", names[v], ms[guidedStage] / 2);
            line += buf;
            if (ms[guidedStage] < best) { best = ms[guidedStage]; bestV = v; }
        }
        setGuidedVariant(bestV);
        if (best < 1e300)
            text += line + " -> " + names[bestV] + "\n";
    }
    lgcr_batch_destroy(b);
    if (report && reportlen) {
        std::strncpy(report, text.c_str(), reportlen - 1);
        report[reportlen - 1] = '\0';
    }
    return status;
}

// Per-batch autotuner: tunes this batch's own launch settings on the given
// items (the layout the caller will run) without touching the process-wide
// settings, so other batches and per-frame calls keep running unchanged:
//  * the block shape of every tunable per-pixel stage the items use
//    (stage-event time of that stage);
//  * the persistent guided kernel's variant (its stage-event time);
//  * the frame grouping of the stage sequence (whole-run time, events around
//    three runs): upscaling frames alone, one group, or one frame per group.
// Later runs of this batch plan with the chosen settings and re-capture their
// graphs.
extern "C" int lgcr_batch_autotune(lgcr_batch *b, const lgcr_batch_item *items, int count,
                                   void *stream, char *report, size_t reportlen) {
    static const int cand[][2] = {{32, 8}, {16, 8}, {32, 4}, {64, 4}, {16, 16}, {128, 2}, {8, 8}};
    static const char *variantNames[3] = {"2-blocks", "3-blocks", "staged"};
    if (!b || !items || count <= 0) {
        setError("LGCR: empty batch");
        return LGCR_E_ARGUMENT;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const bool wasProfiling = b->profiling;
    if (!b->ownConfig) {
        b->cfg = processLaunchConfig();
        b->ownConfig = true;
    }
    if (b->groupMode < -1)
        b->groupMode = batchGroupFrames();
    std::vector<double> ms(stageCount());
    int status = LGCR_OK;
    // one untimed run, then two timed ones: stage times per run
    auto stageRun = [&]() {
        status = lgcr_batch_run(b, items, count, stream, 0);
        lgcr_batch_stage_times(b, nullptr, nullptr, 1);
        for (int rep = 0; rep < 2 && status == LGCR_OK; ++rep)
            status = lgcr_batch_run(b, items, count, stream, 0);
        lgcr_batch_stage_times(b, ms.data(), nullptr, 1);
        for (double &v : ms)
            v /= 2.0;
    };
    std::string text;
    b->profiling = true;
    for (int st = 0; st < stageCount() && status == LGCR_OK; ++st) {
        if (!stageTunable(st))
            continue;
        int bestX = b->cfg.shapeX[st], bestY = b->cfg.shapeY[st];
        double best = 1e300;
        std::string line = std::string(stageName(st)) + ":";
        for (const auto &c : cand) {
            b->cfg.shapeX[st] = c[0];
            b->cfg.shapeY[st] = c[1];
            stageRun();
            if (status != LGCR_OK || ms[st] <= 0.0)
                break;                          // stage not used by these items
            char buf[64];
            std::snprintf(buf, sizeof(buf), " %dx%d=%.3fms", c[0], c[1], ms[st]);
            line += buf;
            if (ms[st] < best) { best = ms[st]; bestX = c[0]; bestY = c[1]; }
        }
        b->cfg.shapeX[st] = bestX;
        b->cfg.shapeY[st] = bestY;
        if (best < 1e300) {
            char buf[48];
            std::snprintf(buf, sizeof(buf), " -> %dx%d\n", bestX, bestY);
            text += line + buf;
        }
    }
    int guidedStage = -1;
    for (int st = 0; st < stageCount(); ++st)
        if (std::string(stageName(st)) == "reconstructChroma")
            guidedStage = st;
    if (status == LGCR_OK && guidedStage >= 0) {
        int bestV = b->cfg.guidedVariant;
        double best = 1e300;
        std::string line = "reconstructChroma:";
        for (int v = 0; v < 3 && status == LGCR_OK; ++v) {
            b->cfg.guidedVariant = v;
            stageRun();
            if (status != LGCR_OK || ms[guidedStage] <= 0.0)
                break;
            char buf[64];
            std::snprintf(buf, sizeof(buf), " %s=%.3fms", variantNames[v], ms[guidedStage]);
            line += buf;
            if (ms[guidedStage] < best) { best = ms[guidedStage]; bestV = v; }
        }
        b->cfg.guidedVariant = bestV;
        if (best < 1e300)
            text += line + " -> " + variantNames[bestV] + "\n";
    }
    // frame grouping: whole runs between events, profiling off
    b->profiling = false;
    if (status == LGCR_OK) {
        cudaEvent_t t0 = nullptr, t1 = nullptr;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        static const int modes[3] = {-1, 0, 1};
        static const char *modeNames[3] = {"upscaling-alone", "one-group", "per-frame"};
        int bestMode = b->groupMode;
        double best = 1e300;
        std::string line = "frame groups:";
        for (int m = 0; m < 3 && status == LGCR_OK; ++m) {
            b->groupMode = modes[m];
            status = lgcr_batch_run(b, items, count, stream, 0);
            cudaEventRecord(t0, s);
            for (int rep = 0; rep < 3 && status == LGCR_OK; ++rep)
                status = lgcr_batch_run(b, items, count, stream, 0);
            cudaEventRecord(t1, s);
            float t = 0.0f;
            if (status != LGCR_OK || cudaEventSynchronize(t1) != cudaSuccess ||
                cudaEventElapsedTime(&t, t0, t1) != cudaSuccess)
                break;
            char buf[64];
            std::snprintf(buf, sizeof(buf), " %s=%.3fms", modeNames[m], t / 3.0);
            line += buf;
            if (t < best) { best = t; bestMode = modes[m]; }
        }
        b->groupMode = bestMode;
        if (best < 1e300)
            text += line + " -> " + modeNames[bestMode == -1 ? 0 : bestMode == 0 ? 1 : 2] + "\n";
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
    }
    b->profiling = wasProfiling;
    ++b->cfgVersion;                    // graphs of earlier settings are re-captured
    if (report && reportlen) {
        std::strncpy(report, text.c_str(), reportlen - 1);
        report[reportlen - 1] = '\0';
    }
    return status;
}
