// serve.cu -- the request loop: admission by device footprint and continuous
// batching on one GPU.
//
// A context owns one device arena.  hm_submit validates a request, sizes its
// footprint (points + outputs + the pipeline scratch hm_workspace_bytes
// plans for it) and queues it.  A scheduler thread forms batches: whenever a
// batch slot (a stream) is free it takes queued requests of one size class in
// arrival order while their footprints fit the arena's largest free block and
// the batch's work cap (small requests go to high-priority streams and never
// wait behind a large request's batch), reserves one block for them, and enqueues on the slot's stream
// the copies in, the whole pipeline (hm_batch_bind + hm_batch_run), the copies
// out and a host callback.  The callback only marks the slot finished; the
// scheduler then reads each request's counters (copied with the results),
// releases the block and forms the next batch from whatever has arrived, so
// up to max_inflight batches overlap on the device.  A request's results do
// not depend on its batch mates: no reduction mixes rows of different jobs.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "hm_internal.cuh"

namespace hm {

// First-fit allocator over one device allocation; blocks are 256-byte
// aligned and neighbouring free blocks are merged.
struct Arena {
    char *base = nullptr;
    size_t capacity = 0, used = 0, peak = 0;
    std::map<size_t, size_t> free_blocks;  // offset -> size

    void init(char *b, size_t cap) {
        base = b;
        capacity = cap;
        free_blocks.clear();
        if (cap) free_blocks[0] = cap;
    }
    size_t largest() const {
        size_t m = 0;
        for (const auto &f : free_blocks) m = std::max(m, f.second);
        return m;
    }
    bool alloc(size_t bytes, size_t *off) {
        bytes = round_up(std::max<size_t>(bytes, 1), 256);
        for (auto it = free_blocks.begin(); it != free_blocks.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes, at = it->first + bytes;
            free_blocks.erase(it);
            if (rest) free_blocks[at] = rest;
            used += bytes;
            peak = std::max(peak, used);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = round_up(std::max<size_t>(bytes, 1), 256);
        used -= bytes;
        auto it = free_blocks.emplace(off, bytes).first;
        auto next = std::next(it);
        if (next != free_blocks.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_blocks.erase(next);
        }
        if (it != free_blocks.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_blocks.erase(it);
            }
        }
    }
};

struct Request {
    hm_job host{};           // as submitted: host pointers
    size_t io_bytes = 0;     // device copies of points and outputs
    size_t ws_bytes = 0;     // pipeline scratch of the request alone
    double work = 0;         // n * n * d
    bool small = true;       // work <= small_work: high-priority batches
    double submit_ms = 0, admit_ms = 0, done_ms = 0;
    int status = HM_ERR_NOT_READY;
    std::string message;
    int path = 0;
    uint64_t batch = 0;
    uint32_t batch_jobs = 0;
    hm_stats stats{};
    bool finished = false;
    size_t footprint() const { return io_bytes + ws_bytes + 4096; }
};

struct Slot {
    hm_ctx *ctx = nullptr;
    cudaStream_t stream = nullptr;
    JobCounters *counters = nullptr;  // page-locked, max_batch_jobs entries
    bool high = false;                // high-priority stream: small requests
    bool busy = false, done = false;
    double done_ms = 0;
    hm_batch *batch = nullptr;
    size_t off = 0, bytes = 0;
    uint64_t seq = 0;
    std::vector<uint64_t> tickets;
};

static size_t io_bytes_of(const hm_job &r) {
    const size_t n = r.n;
    size_t b = round_up(n * r.d * sizeof(float), 256) + 2 * round_up(n * r.k * 4, 256);
    if (r.sigma_out) b += round_up(n * 4, 256);
    if (r.rho_out) b += round_up(n * 4, 256);
    return b;
}

}  // namespace hm

using namespace hm;

struct hm_ctx {
    int device = 0;
    hm_ctx_config cfg{};
    char *arena_mem = nullptr;
    Arena arena;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<uint64_t> pending;
    std::map<uint64_t, Request> reqs;
    uint64_t next_ticket = 1, batch_seq = 0;
    bool stop = false;
    std::thread worker;
    std::chrono::steady_clock::time_point t0;
    hm_ctx_totals totals{};

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace hm {

static void finish(hm_ctx *C, Request &r, int status, const char *msg, double t) {
    r.status = status;
    r.message = msg ? msg : "";
    r.done_ms = t;
    r.finished = true;
    C->totals.finished++;
    if (status != HM_OK) C->totals.failed++;
}

static void CUDART_CB on_batch_done(void *p) {
    Slot *s = static_cast<Slot *>(p);
    hm_ctx *C = s->ctx;
    const double t = C->now_ms();
    {
        std::lock_guard<std::mutex> lk(C->mu);
        s->done = true;
        s->done_ms = t;
    }
    C->cv_sched.notify_one();
}

// Finished slots: results and counters are on the host; record each
// request's status, release the block.  Called with the lock held.
static void retire(hm_ctx *C) {
    bool any = false;
    for (Slot &s : C->slots) {
        if (!s.busy || !s.done) continue;
        for (size_t j = 0; j < s.tickets.size(); ++j) {
            auto it = C->reqs.find(s.tickets[j]);
            if (it == C->reqs.end()) continue;
            Request &r = it->second;
            const int rc = batch_job_result(s.batch, (uint32_t)j, s.counters[j], &r.stats);
            finish(C, r, rc, rc == HM_OK ? nullptr : hm_last_error(), s.done_ms);
        }
        hm_batch_destroy(s.batch);
        s.batch = nullptr;
        C->arena.release(s.off, s.bytes);
        s.tickets.clear();
        s.busy = s.done = false;
        any = true;
    }
    if (any) C->cv_done.notify_all();
}

// Enqueue one batch on slot `si` for the requests in `take` (already removed
// from the queue, block [off, off + bytes) reserved).  Runs without the lock.
static int launch(hm_ctx *C, Slot &s, std::vector<Request *> &take, size_t off, size_t bytes,
                  size_t *exact_bytes) {
    char *blk = C->arena.base + off;
    const uint32_t nj = (uint32_t)take.size();
    std::vector<hm_job> dev(nj);
    size_t o = 0;
    auto carve = [&](size_t b) {
        char *p = blk + o;
        o += round_up(b, 256);
        return p;
    };
    for (uint32_t j = 0; j < nj; ++j) {
        const hm_job &h = take[j]->host;
        hm_job &d = dev[j];
        d = h;
        d.data = reinterpret_cast<const float *>(carve(h.n * h.d * sizeof(float)));
        d.idx_out = reinterpret_cast<uint32_t *>(carve(h.n * h.k * 4));
        d.dist_out = reinterpret_cast<float *>(carve(h.n * h.k * 4));
        d.sigma_out = h.sigma_out ? reinterpret_cast<float *>(carve(h.n * 4)) : nullptr;
        d.rho_out = h.rho_out ? reinterpret_cast<float *>(carve(h.n * 4)) : nullptr;
    }
    hm_batch *B = nullptr;
    HM_TRY(hm_batch_create(dev.data(), nj, &B));
    const size_t ws = hm_batch_workspace_bytes(B);
    *exact_bytes = o + ws;
    if (o + ws > bytes) {  // the per-request estimate fell short: caller re-reserves
        hm_batch_destroy(B);
        return HM_ERR_NOT_READY;
    }
    s.batch = B;
    cudaStream_t st = s.stream;
    for (uint32_t j = 0; j < nj; ++j)
        HM_CUDA_TRY(cudaMemcpyAsync(const_cast<float *>(dev[j].data), take[j]->host.data,
                                    dev[j].n * dev[j].d * sizeof(float), cudaMemcpyHostToDevice, st));
    HM_TRY(hm_batch_bind(B, blk + o, ws, st));
    HM_TRY(hm_batch_run(B, st));
    for (uint32_t j = 0; j < nj; ++j) {
        const hm_job &h = take[j]->host, &d = dev[j];
        HM_CUDA_TRY(cudaMemcpyAsync(h.idx_out, d.idx_out, h.n * h.k * 4, cudaMemcpyDeviceToHost, st));
        HM_CUDA_TRY(cudaMemcpyAsync(h.dist_out, d.dist_out, h.n * h.k * 4, cudaMemcpyDeviceToHost, st));
        if (h.sigma_out)
            HM_CUDA_TRY(cudaMemcpyAsync(h.sigma_out, d.sigma_out, h.n * 4, cudaMemcpyDeviceToHost, st));
        if (h.rho_out)
            HM_CUDA_TRY(cudaMemcpyAsync(h.rho_out, d.rho_out, h.n * 4, cudaMemcpyDeviceToHost, st));
    }
    HM_CUDA_TRY(cudaMemcpyAsync(s.counters, blk + o + batch_counters_offset(B),
                                nj * sizeof(JobCounters), cudaMemcpyDeviceToHost, st));
    HM_CUDA_TRY(cudaLaunchHostFunc(st, on_batch_done, &s));
    for (uint32_t j = 0; j < nj; ++j) take[j]->path = hm_batch_job_path(B, j);
    return HM_OK;
}

// Form and enqueue at most one batch.  Called with the lock held; drops it
// around the CUDA calls.  Returns true when a batch was launched.
static bool try_launch(hm_ctx *C, std::unique_lock<std::mutex> &lk) {
    // a free high-priority slot serves small requests; a free low-priority
    // one large requests first, then small ones
    Slot *slot_hi = nullptr, *slot_lo = nullptr;
    for (Slot &s : C->slots) {
        if (s.busy) continue;
        if (s.high && !slot_hi) slot_hi = &s;
        if (!s.high && !slot_lo) slot_lo = &s;
    }
    if (C->pending.empty() || (!slot_hi && !slot_lo)) return false;
    bool any_small = false, any_large = false;
    for (auto it = C->pending.begin(); it != C->pending.end();) {
        Request &r = C->reqs.at(*it);
        if (r.footprint() > C->arena.capacity) {
            char msg[160];
            snprintf(msg, sizeof msg, "request needs %zu bytes of device memory; the context holds %zu",
                     r.footprint(), C->arena.capacity);
            finish(C, r, HM_ERR_ADMISSION, msg, C->now_ms());
            C->cv_done.notify_all();
            it = C->pending.erase(it);
            continue;
        }
        (r.small ? any_small : any_large) = true;
        ++it;
    }
    Slot *slot = nullptr;
    bool want_small = true;
    if (slot_hi && any_small) {
        slot = slot_hi;
    } else if (slot_lo && any_large) {
        slot = slot_lo;
        want_small = false;
    } else if (slot_lo && any_small) {
        slot = slot_lo;
    } else {
        return false;
    }
    // requests of that class in arrival order, while they fit
    const size_t avail = C->arena.largest();
    std::vector<uint64_t> tickets;
    std::vector<Request *> take;
    size_t need = 0;
    double work = 0;
    for (auto it = C->pending.begin(); it != C->pending.end();) {
        Request &r = C->reqs.at(*it);
        if (r.small != want_small) {
            ++it;
            continue;
        }
        if (!take.empty() && (take.size() >= C->cfg.max_batch_jobs || work + r.work > C->cfg.max_batch_work))
            break;
        if (need + r.footprint() > avail) break;  // arrival order: later requests of the class wait too
        take.push_back(&r);
        tickets.push_back(*it);
        need += r.footprint();
        work += r.work;
        it = C->pending.erase(it);
    }
    if (take.empty()) return false;
    size_t off = 0;
    if (!C->arena.alloc(need, &off)) {  // cannot happen: need <= largest free block
        for (auto it = tickets.rbegin(); it != tickets.rend(); ++it) C->pending.push_front(*it);
        return false;
    }
    const uint64_t seq = ++C->batch_seq;
    const double t_admit = C->now_ms();
    for (Request *r : take) {
        r->admit_ms = t_admit;
        r->batch = seq;
        r->batch_jobs = (uint32_t)take.size();
    }
    slot->busy = true;
    slot->done = false;
    slot->seq = seq;
    slot->off = off;
    slot->bytes = need;
    slot->tickets = tickets;
    C->totals.batches++;
    C->totals.max_batch_jobs_seen = std::max<uint32_t>(C->totals.max_batch_jobs_seen, (uint32_t)take.size());
    uint32_t inflight = 0;
    for (const Slot &s : C->slots) inflight += s.busy ? 1 : 0;
    C->totals.max_inflight_seen = std::max(C->totals.max_inflight_seen, inflight);

    lk.unlock();
    size_t exact = 0;
    int rc = launch(C, *slot, take, off, need, &exact);
    std::string msg = rc == HM_OK ? std::string() : std::string(hm_last_error());
    if (rc != HM_OK && rc != HM_ERR_NOT_READY) cudaStreamSynchronize(slot->stream);  // nothing left in flight
    lk.lock();
    if (rc == HM_OK) return true;
    // not launched: give the block back
    if (slot->batch) {
        hm_batch_destroy(slot->batch);
        slot->batch = nullptr;
    }
    C->arena.release(off, need);
    slot->busy = false;
    slot->tickets.clear();
    C->totals.batches--;
    if (rc == HM_ERR_NOT_READY) {
        // the estimate was short: requeue, and size these requests by the
        // exact batch scratch next time
        const double extra = (double)(exact - need) / take.size();
        for (auto it = take.rbegin(); it != take.rend(); ++it) (*it)->ws_bytes += (size_t)extra + 256;
        for (auto it = tickets.rbegin(); it != tickets.rend(); ++it) C->pending.push_front(*it);
        return true;  // try again at once
    }
    const double t = C->now_ms();
    for (Request *r : take) finish(C, *r, rc, msg.c_str(), t);
    C->cv_done.notify_all();
    return true;
}

static void scheduler(hm_ctx *C) {
    cudaSetDevice(C->device);
    std::unique_lock<std::mutex> lk(C->mu);
    for (;;) {
        retire(C);
        const bool launched = try_launch(C, lk);
        bool busy = false;
        for (const Slot &s : C->slots) busy |= s.busy;
        if (C->stop && C->pending.empty() && !busy) break;
        if (!launched) C->cv_sched.wait_for(lk, std::chrono::milliseconds(2));
    }
}

static void fill_info(const Request &r, hm_request_info *info) {
    if (!info) return;
    memset(info, 0, sizeof *info);
    info->status = r.finished ? r.status : HM_ERR_NOT_READY;
    info->path_used = r.path;
    info->batch = r.batch;
    info->batch_jobs = r.batch_jobs;
    info->submit_ms = r.submit_ms;
    info->admit_ms = r.admit_ms;
    info->done_ms = r.done_ms;
    info->stats = r.stats;
}

static int request_status(const Request &r) {
    if (!r.finished) return HM_ERR_NOT_READY;
    if (r.status != HM_OK) return set_error(r.status, "%s", r.message.c_str());
    return HM_OK;
}

}  // namespace hm

extern "C" {

int hm_ctx_create(const hm_ctx_config *config, hm_ctx **out) {
    clear_error();
    if (!out) return set_error(HM_ERR_INVALID, "NULL output pointer");
    *out = nullptr;
    hm_ctx_config cfg{};
    if (config) cfg = *config;
    if (cfg.max_inflight == 0) cfg.max_inflight = 4;
    if (cfg.max_batch_jobs == 0) cfg.max_batch_jobs = 64;
    if (cfg.max_batch_work <= 0) cfg.max_batch_work = 4e11;
    if (cfg.small_work <= 0) cfg.small_work = 2e10;
    if (cfg.max_inflight > 64) return set_error(HM_ERR_INVALID, "max_inflight above 64");
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    if (cfg.memory_bytes == 0) {
        size_t fr = 0, tot = 0;
        HM_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        cfg.memory_bytes = (fr / 4 * 3) & ~((uint64_t(2) << 20) - 1);
    }
    hm_ctx *C = new (std::nothrow) hm_ctx();
    if (!C) return set_error(HM_ERR_OOM, "host allocation failed");
    C->device = dev;
    C->cfg = cfg;
    C->t0 = std::chrono::steady_clock::now();
    cudaError_t e = cudaMalloc(&C->arena_mem, cfg.memory_bytes);
    if (e != cudaSuccess) {
        delete C;
        return set_error(HM_ERR_OOM, "device arena of %llu bytes: %s", (unsigned long long)cfg.memory_bytes,
                         cudaGetErrorString(e));
    }
    C->arena.init(C->arena_mem, cfg.memory_bytes);
    C->totals.arena_bytes = cfg.memory_bytes;
    C->slots.resize(cfg.max_inflight);
    int prio_lo = 0, prio_hi = 0;
    e = cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    for (size_t i = 0; e == cudaSuccess && i < C->slots.size(); ++i) {
        Slot &s = C->slots[i];
        s.ctx = C;
        s.high = cfg.max_inflight > 1 && i < (cfg.max_inflight + 1) / 2;  // at least one low slot
        e = cudaStreamCreateWithPriority(&s.stream, cudaStreamNonBlocking, s.high ? prio_hi : prio_lo);
        if (e == cudaSuccess)
            e = cudaMallocHost(reinterpret_cast<void **>(&s.counters), cfg.max_batch_jobs * sizeof(JobCounters));
        if (e != cudaSuccess) break;
    }
    if (e != cudaSuccess) {
        for (Slot &s : C->slots) {
            if (s.stream) cudaStreamDestroy(s.stream);
            if (s.counters) cudaFreeHost(s.counters);
        }
        cudaFree(C->arena_mem);
        delete C;
        return set_error(HM_ERR_CUDA, "context set-up: %s", cudaGetErrorString(e));
    }
    C->worker = std::thread(scheduler, C);
    *out = C;
    return HM_OK;
}

int hm_ctx_destroy(hm_ctx *C) {
    clear_error();
    if (!C) return HM_OK;
    {
        std::lock_guard<std::mutex> lk(C->mu);
        C->stop = true;
    }
    C->cv_sched.notify_all();
    if (C->worker.joinable()) C->worker.join();
    for (Slot &s : C->slots) {
        if (s.stream) cudaStreamDestroy(s.stream);
        if (s.counters) cudaFreeHost(s.counters);
    }
    cudaFree(C->arena_mem);
    delete C;
    return HM_OK;
}

int hm_submit(hm_ctx *C, const hm_job *r, uint64_t *ticket) {
    clear_error();
    if (!C || !r || !ticket) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (!r->data || !r->idx_out || !r->dist_out)
        return set_error(HM_ERR_INVALID, "request has a NULL data/output pointer");
    // validates the request and sizes its scratch (host planning only)
    const size_t ws = hm_workspace_bytes(r->n, r->d, r->k, r->metric, r->path);
    if (ws == 0) return HM_ERR_INVALID;  // message set by hm_workspace_bytes
    Request q;
    q.host = *r;
    q.io_bytes = io_bytes_of(*r);
    q.ws_bytes = ws;
    q.work = (double)r->n * (double)r->n * (double)r->d;
    q.small = q.work <= C->cfg.small_work;
    {
        std::lock_guard<std::mutex> lk(C->mu);
        if (C->stop) return set_error(HM_ERR_INVALID, "context is shutting down");
        q.submit_ms = C->now_ms();
        const uint64_t t = C->next_ticket++;
        C->reqs.emplace(t, std::move(q));
        C->pending.push_back(t);
        C->totals.submitted++;
        *ticket = t;
    }
    C->cv_sched.notify_one();
    return HM_OK;
}

int hm_poll(hm_ctx *C, uint64_t ticket, hm_request_info *info) {
    clear_error();
    if (!C) return set_error(HM_ERR_INVALID, "context is NULL");
    std::lock_guard<std::mutex> lk(C->mu);
    auto it = C->reqs.find(ticket);
    if (it == C->reqs.end()) return set_error(HM_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    fill_info(it->second, info);
    return request_status(it->second);
}

int hm_wait(hm_ctx *C, uint64_t ticket, uint64_t timeout_ns, hm_request_info *info) {
    clear_error();
    if (!C) return set_error(HM_ERR_INVALID, "context is NULL");
    // timeouts at or above 2^62 ns (about 146 years; UINT64_MAX included)
    // mean "no deadline": they would overflow the signed clock arithmetic
    const bool forever = timeout_ns >= (1ull << 62);
    const auto deadline = std::chrono::steady_clock::now() +
                          std::chrono::nanoseconds(forever ? 0 : (int64_t)timeout_ns);
    std::unique_lock<std::mutex> lk(C->mu);
    for (;;) {
        auto it = C->reqs.find(ticket);
        if (it == C->reqs.end())
            return set_error(HM_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
        if (it->second.finished || (!forever && std::chrono::steady_clock::now() >= deadline)) {
            fill_info(it->second, info);
            return request_status(it->second);
        }
        if (forever)
            C->cv_done.wait(lk);
        else
            C->cv_done.wait_until(lk, deadline);
    }
}

int hm_release(hm_ctx *C, uint64_t ticket) {
    clear_error();
    if (!C) return set_error(HM_ERR_INVALID, "context is NULL");
    std::lock_guard<std::mutex> lk(C->mu);
    auto it = C->reqs.find(ticket);
    if (it == C->reqs.end()) return set_error(HM_ERR_INVALID, "unknown ticket %llu", (unsigned long long)ticket);
    if (!it->second.finished) return set_error(HM_ERR_NOT_READY, "ticket %llu is still pending",
                                               (unsigned long long)ticket);
    C->reqs.erase(it);
    return HM_OK;
}

int hm_ctx_totals_read(hm_ctx *C, hm_ctx_totals *t) {
    clear_error();
    if (!C || !t) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    std::lock_guard<std::mutex> lk(C->mu);
    *t = C->totals;
    t->arena_peak_bytes = C->arena.peak;
    return HM_OK;
}

}  // extern "C"
