// Serving form: a request loop with continuous batching.
//
// Requests carry host planes. `lanes` worker threads each own a CUDA stream
// and a batch object (device workspaces per slot, graph cache). A lane takes
// up to `max_batch` queued requests whose device footprint fits the
// remaining memory budget, uploads them, runs one batched launch sequence,
// downloads, and completes them; while one lane's batch is on the GPU the
// next requests are admitted by another lane, so their work overlaps on the
// device. Each filter keeps its tables resident; each lane keeps its
// workspaces between batches. All waits are bounded by the caller's timeout
// and report LGCR_E_TIMEOUT / LGCR_E_CLOSED instead of blocking forever.
//
// The reference has no serving loop: VapourSynth calls lgcrGetFrame from
// its worker threads (fmParallel, src/plugin.cpp:1157) with a per-worker
// workspace pool sized by the thread count (src/plugin.cpp:215-217,
// src/workspace.cpp:83-120); this form replaces that scheduling.
#include "impl.h"

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

using namespace lgcr_b200;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t ticket = 0;
    lgcr_recon *filter = nullptr;
    lgcr_plane in[3], out[3];
    int chromaLocation = -1;
    size_t cost = 0;
    int status = LGCR_OK;
    bool done = false;
    double submitMs = 0, startMs = 0, doneMs = 0;
    int batchSize = 0;
};

// Staging planes of one batch position of a lane. They grow to the largest
// frame the position has seen, in stream order on the lane's stream: a
// stream-ordered free and allocation do not synchronize the device, so a
// mixed stream growing its slots never stalls the other lanes' batches.
struct DeviceSlot {
    cudaStream_t stream = nullptr;
    void *in[3] = {nullptr, nullptr, nullptr};
    void *out[3] = {nullptr, nullptr, nullptr};
    size_t inBytes[3] = {0, 0, 0}, outBytes[3] = {0, 0, 0};
    explicit DeviceSlot(cudaStream_t s) : stream(s) {}
    ~DeviceSlot() {
        for (int i = 0; i < 3; ++i) {
            if (in[i]) cudaFreeAsync(in[i], stream);
            if (out[i]) cudaFreeAsync(out[i], stream);
        }
    }
    bool ensure(int p, bool isIn, size_t bytes) {
        void *&ptr = isIn ? in[p] : out[p];
        size_t &have = isIn ? inBytes[p] : outBytes[p];
        if (have >= bytes)
            return true;
        if (ptr) cudaFreeAsync(ptr, stream);
        ptr = nullptr;
        have = 0;
        if (cudaMallocAsync(&ptr, bytes, stream) != cudaSuccess)
            return false;
        have = bytes;
        return true;
    }
};

} // namespace

struct lgcr_server {
    lgcr_server_config cfg{};
    std::mutex mu;
    std::condition_variable queued, finished;
    std::deque<Request *> queue;
    std::unordered_map<int64_t, std::unique_ptr<Request>> requests;
    int64_t nextTicket = 0;
    size_t inUse = 0;
    bool running = true;
    bool paused = false;
    std::vector<std::thread> lanes;
    Clock::time_point t0 = Clock::now();
    int device = 0;
    double now() const {
        return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    }
};

namespace {

size_t planeBytes(const lgcr_plane &p, int bps) { return size_t(p.width) * p.height * bps; }

// Device footprint of one request: staging planes plus its frame workspace.
size_t requestCost(lgcr_recon *f, const lgcr_plane *in, const lgcr_plane *out) {
    Filter &F = *f->filter;
    const int bps = F.bytesPerSample();
    size_t bytes = 0;
    for (int i = 0; i < 3; ++i) {
        bytes += planeBytes(in[i], bps);
        if (out[i].data) bytes += planeBytes(out[i], bps);
    }
    const size_t L = size_t(F.sw) * F.sh, C = size_t(F.cw) * F.ch, O = size_t(F.p.outW) * F.p.outH;
    // converted planes, tensor, masks, float outputs, algo workspaces (upper bound)
    bytes += 4 * (L + 2 * C) + 12 * L + 4 * L + 8 * O + 4 * (9 * C + 2 * L + O);
    return bytes;
}

void laneLoop(lgcr_server *S, int laneIndex) {
    cudaSetDevice(S->device);
    cudaStream_t stream = nullptr;
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    lgcr_batch *batch = nullptr;
    lgcr_batch_create(&batch);
    std::vector<std::unique_ptr<DeviceSlot>> slots;
    (void)laneIndex;
    for (;;) {
        std::vector<Request *> take;
        size_t reserved = 0;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            S->queued.wait(lock, [&] { return !S->running || (!S->paused && !S->queue.empty()); });
            if (!S->running)
                break;
            // admit from the front while the budget allows (at least one)
            while (!S->queue.empty() && (int)take.size() < S->cfg.max_batch) {
                Request *r = S->queue.front();
                if (!take.empty() && S->inUse + reserved + r->cost > S->cfg.device_budget_bytes)
                    break;
                if (take.empty() && S->inUse + r->cost > S->cfg.device_budget_bytes && S->inUse > 0)
                    break;                    // wait for running batches to free memory
                S->queue.pop_front();
                take.push_back(r);
                reserved += r->cost;
            }
            if (take.empty()) {
                S->queued.wait_for(lock, std::chrono::milliseconds(5));
                continue;
            }
            S->inUse += reserved;
            const double start = S->now();
            for (Request *r : take) {
                r->startMs = start;
                r->batchSize = int(take.size());
            }
        }
        // upload, run, download
        int status = LGCR_OK;
        if (slots.size() < take.size())
            slots.resize(take.size());
        std::vector<lgcr_batch_item> items(take.size());
        for (size_t i = 0; i < take.size() && status == LGCR_OK; ++i) {
            Request *r = take[i];
            if (!slots[i]) slots[i] = std::make_unique<DeviceSlot>(stream);
            const int bps = r->filter->filter->bytesPerSample();
            items[i].filter = r->filter;
            items[i].chroma_location = r->chromaLocation;
            for (int p = 0; p < 3; ++p) {
                const size_t inRow = size_t(r->in[p].width) * bps;
                if (!slots[i]->ensure(p, true, inRow * r->in[p].height)) { status = LGCR_E_NOMEM; break; }
                if (copyPlane(slots[i]->in[p], inRow, r->in[p].data, r->in[p].stride, inRow,
                              r->in[p].height, cudaMemcpyHostToDevice, stream) != cudaSuccess) {
                    status = LGCR_E_CUDA; break;
                }
                items[i].in[p] = { slots[i]->in[p], (ptrdiff_t)inRow, r->in[p].width, r->in[p].height };
                if (r->out[p].data) {
                    const size_t outRow = size_t(r->out[p].width) * bps;
                    if (!slots[i]->ensure(p, false, outRow * r->out[p].height)) { status = LGCR_E_NOMEM; break; }
                    items[i].out[p] = { slots[i]->out[p], (ptrdiff_t)outRow, r->out[p].width, r->out[p].height };
                } else {
                    items[i].out[p] = { nullptr, 0, r->out[p].width, r->out[p].height };
                }
            }
        }
        if (status == LGCR_OK)
            status = lgcr_batch_run(batch, items.data(), int(items.size()), stream, 0);
        for (size_t i = 0; i < take.size() && status == LGCR_OK; ++i) {
            Request *r = take[i];
            const int bps = r->filter->filter->bytesPerSample();
            for (int p = 0; p < 3; ++p) {
                if (!r->out[p].data)
                    continue;
                const size_t outRow = size_t(r->out[p].width) * bps;
                if (copyPlane(r->out[p].data, r->out[p].stride, slots[i]->out[p], outRow, outRow,
                              r->out[p].height, cudaMemcpyDeviceToHost, stream) != cudaSuccess) {
                    status = LGCR_E_CUDA; break;
                }
            }
        }
        if (cudaStreamSynchronize(stream) != cudaSuccess && status == LGCR_OK)
            status = LGCR_E_CUDA;
        {
            std::lock_guard<std::mutex> lock(S->mu);
            const double end = S->now();
            for (Request *r : take) {
                r->status = status;
                r->doneMs = end;
                r->done = true;
            }
            S->inUse -= reserved;
        }
        S->finished.notify_all();
        S->queued.notify_all();
    }
    lgcr_batch_destroy(batch);
    slots.clear();
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
}

} // namespace

extern "C" {

int lgcr_server_create(const lgcr_server_config *config, lgcr_server **out) {
    if (!config || !out || config->max_batch < 1 || config->lanes < 1 || config->queue_capacity < 1 ||
        config->device_budget_bytes == 0) {
        setError("LGCR: invalid server configuration");
        return LGCR_E_ARGUMENT;
    }
    auto S = std::make_unique<lgcr_server>();
    S->cfg = *config;
    cudaGetDevice(&S->device);
    for (int i = 0; i < config->lanes; ++i)
        S->lanes.emplace_back(laneLoop, S.get(), i);
    *out = S.release();
    return LGCR_OK;
}

int64_t lgcr_server_submit(lgcr_server *S, lgcr_recon *filter, const lgcr_plane in[3],
                           const lgcr_plane out[3], int chroma_location) {
    if (!S || !filter || !in || !out)
        return -LGCR_E_ARGUMENT;
    auto r = std::make_unique<Request>();
    r->filter = filter;
    for (int i = 0; i < 3; ++i) {
        r->in[i] = in[i];
        r->out[i] = out[i];
    }
    r->chromaLocation = chroma_location;
    r->cost = requestCost(filter, in, out);
    std::lock_guard<std::mutex> lock(S->mu);
    if (!S->running)
        return -LGCR_E_CLOSED;
    if (r->cost > S->cfg.device_budget_bytes) {
        setError("LGCR: request exceeds the server's device-memory budget");
        return -LGCR_E_BUSY;
    }
    if ((int)S->queue.size() >= S->cfg.queue_capacity) {
        setError("LGCR: server queue is full");
        return -LGCR_E_BUSY;
    }
    r->ticket = S->nextTicket++;
    r->submitMs = S->now();
    Request *raw = r.get();
    S->requests.emplace(raw->ticket, std::move(r));
    S->queue.push_back(raw);
    S->queued.notify_one();
    return raw->ticket;
}

int lgcr_server_wait(lgcr_server *S, int64_t ticket, int timeout_ms, lgcr_request_info *info) {
    if (!S)
        return LGCR_E_ARGUMENT;
    std::unique_lock<std::mutex> lock(S->mu);
    auto it = S->requests.find(ticket);
    if (it == S->requests.end())
        return LGCR_E_ARGUMENT;
    Request *r = it->second.get();
    auto ready = [&] { return r->done || !S->running; };
    if (timeout_ms < 0)
        S->finished.wait(lock, ready);
    else if (!S->finished.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready))
        return LGCR_E_TIMEOUT;
    if (!r->done)
        return LGCR_E_CLOSED;
    if (info) {
        info->status = r->status;
        info->submit_ms = r->submitMs;
        info->start_ms = r->startMs;
        info->done_ms = r->doneMs;
        info->batch_size = r->batchSize;
    }
    const int status = r->status;
    S->requests.erase(it);
    return status;
}

// Hold (on != 0) or release the lanes: queued requests are not admitted
// while held. Used to exercise bounded waits and admission from the host.
int lgcr_server_pause(lgcr_server *S, int on) {
    if (!S)
        return LGCR_E_ARGUMENT;
    {
        std::lock_guard<std::mutex> lock(S->mu);
        S->paused = on != 0;
    }
    S->queued.notify_all();
    return LGCR_OK;
}

void lgcr_server_destroy(lgcr_server *S) {
    if (!S)
        return;
    {
        std::lock_guard<std::mutex> lock(S->mu);
        S->running = false;
        for (Request *r : S->queue) {
            r->status = LGCR_E_CLOSED;
            r->done = true;
        }
        S->queue.clear();
    }
    S->queued.notify_all();
    S->finished.notify_all();
    for (auto &t : S->lanes)
        t.join();
    delete S;
}

} // extern "C"
