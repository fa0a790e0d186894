// Commit server: a request loop with continuous batching (included at the end of pil2_b200.cu).
//
// Requests (host row-major traces) arrive at any time.  A worker thread admits them whenever a
// slot is free and the device-memory budget holds the request's buffers (trace, scratch, LDE,
// tree), and turns them into units of work:
//   * the small requests waiting together (LDE of at most `small_elems` elements each) become one
//     batched unit: one batch::Plan over all of them, so their transposes, NTT windows, leaf sponge
//     and tree levels run as shared grouped launches and a persistent leaf kernel;
//   * a larger request is a plain unit: the single-instance commit.
// Units are admitted while earlier ones run: each unit's host-to-device copy overlaps the kernels
// of the units ahead of it, and each unit's kernels follow the previous unit's on the device.  All
// host-to-device copies go through one copy stream in admission order, so the next unit's trace
// has the whole PCIe link (copies of different streams would share it and all land late).  A
// plain unit's trace crosses in column blocks and each block is extended as soon as it lands (the
// pipeline of commit_witness), so a request that finds the device idle waits for its first
// block's copy, not its whole trace.
// Measured on a B200 with the C3 size mix, letting the units' kernels interleave instead (streams
// of different priorities, no ordering) doubled the median latency at 5 requests/s and lowered the
// throughput at 20 requests/s by 7 %: every kernel here fills the GPU, and co-resident commits only
// slow each other down.  Small requests may overtake waiting large ones — a batched unit is
// admitted ahead of the queue head — but a request is overtaken at most `max_overtakes` times, so
// none waits forever.  Completion is observed through an event per unit; the LDE and the tree of
// every request stay resident on the device (for later query reads) until the caller releases the
// request.  Device buffers come from one device allocation of the budget, made when the server is
// created and carved by a host-side best-fit arena: a request takes two blocks, [trace | scratch]
// returned when its unit completes and [LDE | tree] returned when the caller releases it.  Carving
// is host bookkeeping of a few microseconds; a stream-ordered memory pool measured 25-30 ms per
// allocation for this size mix, which at 20 requests/s left the GPU idle ~20 % of the time while
// requests waited.  No call blocks on the GPU except b200_server_wait_all, whose wait is bounded
// by its timeout.
//
// Mode 0 (b200_server_configure) is the plain FIFO: every request a plain unit in arrival order;
// kept as the comparison point.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <unordered_map>

#include "arena.h"
#include "batch.cuh"

namespace serve {

static double now_ms()
{
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t id = 0;
    const uint64_t *trace = nullptr;
    uint32_t nBits = 0, nBitsExt = 0, nCols = 0, arity = 4;
    uint64_t *root_out = nullptr;
    uint64_t words_trace = 0, words_lde = 0, words_tree = 0;
    uint64_t *d_trace = nullptr, *d_scratch = nullptr, *d_lde = nullptr, *d_tree = nullptr;
    uint64_t root[4] = {0, 0, 0, 0};
    int status = 0;  // 0 queued, 1 running, 2 done, < 0 error
    bool released = false;
    cudaStream_t stream = nullptr;  // the stream its buffers were last used on
    double t_submit = 0, t_admit = 0, t_done = 0;
    // device timeline of its unit, ms since the server's reference event: copies issued (the unit
    // reached its stream), host-to-device copies done, kernels started (copies done and the
    // previous unit finished), kernels done
    double g_issued = -1, g_copied = -1, g_start = -1, g_done = -1;
    uint32_t overtaken = 0;  // times a batch of smaller requests was admitted ahead of it
    bool waited_for_block = false;  // once found no contiguous block of the budget free
    std::string err;  // reason of a failed request (reported to the caller by status())
    uint64_t bytes() const { return 8 * (2 * words_trace + words_lde + words_tree); }
    uint64_t elems() const { return (uint64_t)nCols << nBitsExt; }
};

// One admitted unit of work on one slot: a plain request or a batch of small ones.
struct Unit {
    std::vector<Request *> reqs;
    bool batched = false;
    int slot = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaEvent_t issued = nullptr, copied = nullptr, started = nullptr;  // timeline (timing enabled, like done)
    batch::Plan *plan = nullptr;
};

constexpr size_t STAGING_BYTES = 1u << 20;  // per slot: a batched unit's tables and roots (pinned)

// The budget as one device allocation, carved by a BlockMap (arena.h).  Host bookkeeping only: the
// caller returns a block once no queued or running work uses it.
class Arena {
  public:
    uint64_t *base = nullptr;

    int init(uint64_t bytes)
    {
        const uint64_t words = (bytes + 255) / 256 * BlockMap::UNIT;
        if (cudaMalloc((void **)&base, 8 * words) != cudaSuccess) {
            cudaGetLastError();
            base = nullptr;
            return set_err(B200_ENOMEM, "commit server: the device-memory budget could not be reserved");
        }
        map.reset(words);
        return B200_OK;
    }
    ~Arena()
    {
        if (base) cudaFree(base);
    }
    uint64_t *take(uint64_t w)
    {
        const uint64_t off = map.take(w);
        return off == BlockMap::NONE ? nullptr : base + off;
    }
    void give(uint64_t *p, uint64_t w)
    {
        if (p) map.give((uint64_t)(p - base), w);
    }

  private:
    BlockMap map;
};

class Server {
  public:
    int device = 0, sms = 148;
    uint64_t budget = 0, used = 0;
    int mode = 1;                          // 1 continuous batching, 0 FIFO
    uint64_t small_elems = 1ull << 26;     // batched when NExt * nCols is at most this
    uint32_t max_batch = 64;               // requests per batched unit
    uint32_t max_overtakes = 4;            // times a waiting request may be overtaken by a batch
    std::vector<cudaStream_t> streams;     // [slot]
    cudaStream_t copy_stream = nullptr;                // every unit's host-to-device copies, in admission order
    std::vector<std::vector<cudaEvent_t>> block_events;  // [slot] one per column block of a plain unit
    std::vector<unsigned char *> staging;            // [slot] pinned
    std::vector<unsigned char *> d_tables;           // [slot] device copy of a batched unit's tables
    std::vector<uint64_t *> h_roots;                 // [slot] pinned, plain units' root
    std::vector<int> slot_busy;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request *> queue;
    std::vector<Unit *> running;
    std::unordered_map<int64_t, Request *> all;
    int64_t next_id = 1;
    bool stop = false, configured = false;
    std::thread worker;
    Arena arena;
    cudaEvent_t last_done = nullptr;  // completion of the most recently admitted unit
    cudaEvent_t t0_event = nullptr;   // device-time origin of the request timelines
    std::vector<cudaEvent_t> spare_events;
    int family = 2;                   // hash family of this server's commits (fixed at creation)
    uint64_t units_plain = 0, units_batched = 0, batched_requests = 0, overtakes = 0;
    uint64_t deferred = 0;  // requests that fit the budget but once found no contiguous block, and waited
    double launch_ms = 0;   // host time spent enqueueing units (allocations, copies, kernel launches)
    double alloc_ms = 0;    // the part of it spent in the allocations
    double t_start = 0;

    int start(int dev, uint64_t budget_bytes, uint32_t slots)
    {
        device = dev;
        budget = budget_bytes;
        t_start = now_ms();
        CK(cudaSetDevice(dev), "cudaSetDevice");
        int rc = ensure_init_current();
        if (rc) return rc;
        if ((rc = batch_kernel_attrs())) return rc;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if ((rc = arena.init(budget + (1u << 20)))) return rc;  // slack for the blocks' alignment
        for (uint32_t i = 0; i < slots; i++) {
            cudaStream_t s;
            CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
            streams.push_back(s);
            block_events.emplace_back();
            unsigned char *st = nullptr;
            uint64_t *hr = nullptr;
            CK(cudaMallocHost((void **)&st, STAGING_BYTES), "pinned staging");
            staging.push_back(st);
            unsigned char *dt = nullptr;
            CK(cudaMalloc((void **)&dt, STAGING_BYTES), "batched tables");
            d_tables.push_back(dt);
            CK(cudaMallocHost((void **)&hr, 32), "pinned root");
            h_roots.push_back(hr);
            slot_busy.push_back(0);
        }
        CK(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking), "stream");
        CK(cudaEventCreate(&t0_event), "event");
        CK(cudaEventRecord(t0_event, streams[0]), "event record");
        worker = std::thread([this] { loop(); });
        return B200_OK;
    }

    ~Server()
    {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        if (worker.joinable()) worker.join();
        cudaSetDevice(device);
        if (copy_stream) cudaStreamSynchronize(copy_stream);
        for (cudaStream_t s : streams) cudaStreamSynchronize(s);
        for (Unit *u : running) finish_unit(u, cudaEventQuery(u->done) == cudaSuccess);
        for (auto &kv : all) {
            Request *r = kv.second;
            free_buffers(r);
            delete r;
        }
        cudaDeviceSynchronize();
        for (cudaStream_t s : streams) cudaStreamDestroy(s);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        for (auto &v : block_events)
            for (cudaEvent_t e : v) cudaEventDestroy(e);
        for (unsigned char *p : staging) cudaFreeHost(p);
        for (unsigned char *p : d_tables) cudaFree(p);
        for (uint64_t *p : h_roots) cudaFreeHost(p);
        for (cudaEvent_t e : spare_events) cudaEventDestroy(e);
        if (t0_event) cudaEventDestroy(t0_event);
    }

    // [trace | scratch] back to the arena (the unit's work on it is complete)
    void free_trace(Request *r)
    {
        arena.give(r->d_trace, 2 * r->words_trace);
        r->d_trace = r->d_scratch = nullptr;
    }

    // both blocks of a request (d_scratch and d_tree point into them)
    void free_buffers(Request *r)
    {
        free_trace(r);
        arena.give(r->d_lde, r->words_lde + r->words_tree);
        r->d_lde = r->d_tree = nullptr;
    }

    int64_t submit(const uint64_t *trace, uint32_t nBits, uint32_t nBitsExt, uint32_t nCols, uint32_t arity,
                   uint64_t *root_out)
    {
        auto *r = new Request();
        r->trace = trace;
        r->nBits = nBits;
        r->nBitsExt = nBitsExt;
        r->nCols = nCols;
        r->arity = arity;
        r->root_out = root_out;
        r->words_trace = (1ull << nBits) * nCols;
        r->words_lde = (1ull << nBitsExt) * nCols;
        r->words_tree = merkle::tree_num_elements(1ull << nBitsExt, arity);
        r->t_submit = now_ms();
        {
            std::lock_guard<std::mutex> lk(mu);
            if (r->bytes() > budget) {
                delete r;
                return B200_EBUSY;
            }
            r->id = next_id++;
            all[r->id] = r;
            queue.push_back(r);
            configured = true;
        }
        cv.notify_all();
        return r->id;
    }

    // A request's two blocks, or none (and the admission waits for blocks to come back)
    bool alloc_request(Request *r)
    {
        const double t = now_ms();
        r->d_trace = arena.take(2 * r->words_trace);
        r->d_lde = r->d_trace ? arena.take(r->words_lde + r->words_tree) : nullptr;
        alloc_ms += now_ms() - t;
        if (!r->d_lde) {
            free_buffers(r);
            if (!r->waited_for_block) deferred++;
            r->waited_for_block = true;
            return false;
        }
        r->d_scratch = r->d_trace + r->words_trace;
        r->d_tree = r->d_lde + r->words_lde;
        return true;
    }

    cudaEvent_t take_event()
    {
        if (!spare_events.empty()) {
            cudaEvent_t e = spare_events.back();
            spare_events.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        return e;
    }

    // Enqueue a unit's copies and kernels on its stream; returns 0 or a B200 error code.
    int launch_unit(Unit *u)
    {
        cudaStream_t s = u->stream;
        if (!(u->issued = take_event()) || cudaEventRecord(u->issued, s) != cudaSuccess) return B200_ECUDA;
        if (!(u->copied = take_event()) || !(u->started = take_event())) return B200_ECUDA;
        if (!u->batched) {
            // column blocks on the copy stream once the buffers are allocated (u->issued, on s), the
            // kernels on s after the unit ahead (last_done)
            Request *r = u->reqs[0];
            r->stream = s;
            PipeBuffers pb;
            pb.staging = r->d_trace;
            pb.cm1 = pb.scratch = r->d_scratch;
            pb.lde = r->d_lde;
            pb.tree = r->d_tree;
            pb.h_root = h_roots[u->slot];
            const bool idle = !last_done || cudaEventQuery(last_done) == cudaSuccess;
            int rc = pipelined_commit(r->trace, r->nBits, r->nBitsExt, r->nCols, r->arity, family, pb,
                                      copy_stream, s, block_events[u->slot], u->copied, u->issued, last_done,
                                      idle, u->started);
            if (rc) return rc;
        } else {
            // small traces: whole copies on the copy stream (after the allocations), then the batched
            // kernels on s after the unit ahead
            if (cudaStreamWaitEvent(copy_stream, u->issued, 0) != cudaSuccess) return B200_ECUDA;
            for (Request *r : u->reqs) {
                r->stream = s;
                if (r->words_trace && cudaMemcpyAsync(r->d_trace, r->trace, 8 * r->words_trace,
                                                      cudaMemcpyHostToDevice, copy_stream) != cudaSuccess)
                    return B200_ECUDA;
            }
            if (cudaEventRecord(u->copied, copy_stream) != cudaSuccess) return B200_ECUDA;
            if (cudaStreamWaitEvent(s, u->copied, 0) != cudaSuccess) return B200_ECUDA;
            if (last_done && cudaStreamWaitEvent(s, last_done, 0) != cudaSuccess) return B200_ECUDA;
            if (cudaEventRecord(u->started, s) != cudaSuccess) return B200_ECUDA;
            std::vector<batch::Inst> in;
            for (Request *r : u->reqs)
                in.push_back(batch::Inst{r->d_trace, r->d_scratch, r->d_lde, r->d_tree, r->nBits, r->nBitsExt,
                                         r->nCols, r->arity});
            u->plan = new batch::Plan();
            u->plan->borrowed = true;
            if (!u->plan->build(in, sms, family)) return set_err(B200_EINVAL, "batched unit: unsupported shape");
            const size_t tbytes = (u->plan->table.size() + 255) & ~size_t(255);
            if (tbytes + 32 * (u->reqs.size() + 1) > STAGING_BYTES)
                return set_err(B200_EINVAL, "batched unit: descriptor tables above the staging size");
            unsigned char *st = staging[u->slot];
            memcpy(st, u->plan->table.data(), u->plan->table.size());
            if (cudaMemcpyAsync(d_tables[u->slot], st, u->plan->table.size(), cudaMemcpyHostToDevice, s) !=
                cudaSuccess)
                return B200_ECUDA;
            u->plan->d_table = d_tables[u->slot];
            u->plan->h_roots = (uint64_t *)(st + tbytes);
            if (u->plan->enqueue(s) != cudaSuccess) return B200_ECUDA;
        }
        if (!(u->done = take_event()) || cudaEventRecord(u->done, s) != cudaSuccess) return B200_ECUDA;
        last_done = u->done;
        return B200_OK;
    }

    void release_events(Unit *u)
    {
        for (cudaEvent_t e : {u->issued, u->copied, u->started, u->done})
            if (e) spare_events.push_back(e);
        u->issued = u->copied = u->started = u->done = nullptr;
    }

    double since_t0(cudaEvent_t e) const
    {
        float ms = -1.0f;
        if (!e || cudaEventElapsedTime(&ms, t0_event, e) != cudaSuccess) {
            cudaGetLastError();
            return -1.0;
        }
        return (double)ms;
    }

    int free_slot() const
    {
        for (size_t i = 0; i < slot_busy.size(); i++)
            if (!slot_busy[i]) return (int)i;
        return -1;
    }

    // One admission round (caller holds mu): while a slot is free, the next unit holds the waiting
    // small requests (in arrival order, up to max_batch; a batch when there are several), passing
    // the large requests between them unless one of those has been overtaken max_overtakes times;
    // with no small request waiting, the queue head.  Stops at the first unit the budget cannot hold
    // or the arena has no blocks for (the next completion or release retries).
    void admit()
    {
        while (!queue.empty()) {
            const int slot = free_slot();
            if (slot < 0) return;
            auto *u = new Unit();
            u->slot = slot;
            uint64_t add = 0;
            if (mode == 1) {
                std::vector<size_t> small;
                for (size_t i = 0; i < queue.size() && small.size() < max_batch; i++) {
                    Request *r = queue[i];
                    if (r->elems() <= small_elems) {
                        if (used + add + r->bytes() > budget || !alloc_request(r)) break;
                        small.push_back(i);
                        add += r->bytes();
                    } else if (r->overtaken >= max_overtakes) {
                        break;  // this one goes next: nothing behind it passes it again
                    }
                }
                if (!small.empty()) {
                    for (size_t i = 0; i < small.back(); i++)
                        if (queue[i]->elems() > small_elems) {
                            queue[i]->overtaken++;
                            overtakes++;
                        }
                    for (size_t k = small.size(); k-- > 0;) {
                        u->reqs.insert(u->reqs.begin(), queue[small[k]]);
                        queue.erase(queue.begin() + (std::ptrdiff_t)small[k]);
                    }
                } else {
                    add = 0;
                }
            }
            if (u->reqs.empty()) {
                Request *head = queue.front();
                if (used + head->bytes() > budget || !alloc_request(head)) {
                    delete u;
                    return;
                }
                queue.pop_front();
                add = head->bytes();
                u->reqs.push_back(head);
            }
            u->batched = u->reqs.size() > 1;
            u->stream = streams[slot];
            const double t = now_ms();
            for (Request *r : u->reqs) r->t_admit = t;
            const double t_launch = now_ms();
            int rc = launch_unit(u);
            launch_ms += now_ms() - t_launch;
            if (rc) {
                // whatever was enqueued before the failure finishes before the blocks are reused
                cudaStreamSynchronize(copy_stream);
                cudaStreamSynchronize(u->stream);
                cudaGetLastError();
                for (Request *r : u->reqs) {
                    free_buffers(r);
                    if (r->err.empty()) r->err = "request failed on the device (CUDA error)";
                    r->status = rc;
                    r->t_done = now_ms();
                }
                release_events(u);
                delete u->plan;
                delete u;
                continue;
            }
            used += add;
            slot_busy[slot] = 1;
            for (Request *r : u->reqs) r->status = 1;
            if (u->batched) {
                units_batched++;
                batched_requests += u->reqs.size();
            } else {
                units_plain++;
            }
            running.push_back(u);
        }
    }

    // results of a finished unit to its requests; frees the unit (caller holds mu)
    void finish_unit(Unit *u, bool ok)
    {
        const double t = now_ms();
        const double gi = ok ? since_t0(u->issued) : -1, gc = ok ? since_t0(u->copied) : -1,
                     gs = ok ? since_t0(u->started) : -1, gd = ok ? since_t0(u->done) : -1;
        for (size_t i = 0; i < u->reqs.size(); i++) {
            Request *r = u->reqs[i];
            r->t_done = t;
            r->g_issued = gi;
            r->g_copied = gc;
            r->g_start = gs;
            r->g_done = gd;
            if (ok) {
                const uint64_t *src = u->batched ? u->plan->h_roots + 4 * i : h_roots[u->slot];
                memcpy(r->root, src, 32);
                if (r->root_out) memcpy(r->root_out, r->root, 32);
                r->status = 2;
                free_trace(r);  // the unit's kernels are done with the trace and the scratch
                used -= 8 * 2 * r->words_trace;
            } else {
                r->status = B200_ECUDA;
                r->err = "request failed on the device (CUDA error)";
                free_buffers(r);
                used -= r->bytes();
            }
        }
        if (last_done == u->done) last_done = nullptr;
        release_events(u);
        slot_busy[u->slot] = 0;
        delete u->plan;
        delete u;
    }

    // caller holds mu
    void harvest()
    {
        for (size_t i = 0; i < running.size();) {
            Unit *u = running[i];
            const cudaError_t q = cudaEventQuery(u->done);
            if (q == cudaErrorNotReady) {
                i++;
                continue;
            }
            running[i] = running.back();
            running.pop_back();
            finish_unit(u, q == cudaSuccess);
        }
    }

    void loop()
    {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lk(mu);
        while (!stop) {
            harvest();
            admit();
            cv.notify_all();
            cv.wait_for(lk, std::chrono::microseconds(running.empty() ? 2000 : 50));
        }
    }

    int status(int64_t id, double *latency_ms)
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = all.find(id);
        if (it == all.end()) return set_err(B200_EINVAL, "unknown request id");
        Request *r = it->second;
        if (r->status == 2 || r->status < 0) {
            if (latency_ms) *latency_ms = r->t_done - r->t_submit;
            if (r->status < 0) return set_err(r->status, "request " + std::to_string(id) + ": " + r->err);
            return 1;
        }
        return 0;
    }

    int wait_all(uint64_t timeout_ms)
    {
        std::unique_lock<std::mutex> lk(mu);
        const double deadline = now_ms() + (double)timeout_ms;
        while (!queue.empty() || !running.empty()) {
            if (now_ms() > deadline) return set_err(B200_ETIMEOUT, "b200_server_wait_all: timeout");
            cv.wait_for(lk, std::chrono::milliseconds(1));
        }
        return B200_OK;
    }

    int release(int64_t id)
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = all.find(id);
        if (it == all.end()) return set_err(B200_EINVAL, "unknown request id");
        Request *r = it->second;
        if (r->status != 2 && r->status >= 0) return set_err(B200_EBUSY, "request still in flight");
        if (!r->released) {
            cudaSetDevice(device);
            free_buffers(r);
            if (r->status == 2) used -= 8 * (r->words_lde + r->words_tree);
            r->released = true;
        }
        cv.notify_all();
        return B200_OK;
    }
};

}  // namespace serve

extern "C" void *b200_server_new(int device, uint64_t budget_bytes, uint32_t slots)
{
    if (slots == 0 || slots > 64) {
        set_err(B200_EINVAL, "slots must be 1..64");
        return nullptr;
    }

    auto *s = new serve::Server();
    s->family = g_native_family.load();
    if (s->start(device, budget_bytes, slots)) {
        delete s;
        return nullptr;
    }
    return s;
}

extern "C" int b200_server_configure(void *srv, int batching, uint64_t small_elems, uint32_t max_batch)
{
    auto *s = (serve::Server *)srv;
    if (!s) return set_err(B200_EINVAL, "null server");
    if (batching != 0 && batching != 1) return set_err(B200_EINVAL, "batching must be 0 (FIFO) or 1");
    if (max_batch == 0 || max_batch > 1024) return set_err(B200_EINVAL, "max_batch must be 1..1024");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->configured) return set_err(B200_EBUSY, "b200_server_configure: requests already submitted");
    s->mode = batching;
    s->small_elems = small_elems;
    s->max_batch = max_batch;
    return B200_OK;
}

// counters, in this order: plain units, batched units, requests in batched units, requests that
// fit the budget but once found no contiguous block in it (and waited for one), times a waiting request
// was passed, microseconds the worker spent enqueueing units (allocations included), microseconds
// of that in allocations
extern "C" int b200_server_stats(void *srv, uint64_t *out, uint64_t n)
{
    auto *s = (serve::Server *)srv;
    if (!s || (n && !out)) return set_err(B200_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    const uint64_t v[7] = {s->units_plain, s->units_batched, s->batched_requests, s->deferred, s->overtakes,
                           (uint64_t)((s->launch_ms + s->alloc_ms) * 1e3), (uint64_t)(s->alloc_ms * 1e3)};
    for (uint64_t i = 0; i < n && i < 7; i++) out[i] = v[i];
    return B200_OK;
}

// submission, admission and completion time of a request, ms since the server was created
extern "C" int b200_server_request_times(void *srv, int64_t id, double *times3)
{
    auto *s = (serve::Server *)srv;
    if (!s || !times3) return set_err(B200_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return set_err(B200_EINVAL, "unknown request id");
    const serve::Request *r = it->second;
    times3[0] = r->t_submit - s->t_start;
    times3[1] = r->t_admit ? r->t_admit - s->t_start : -1;
    times3[2] = r->t_done ? r->t_done - s->t_start : -1;
    return B200_OK;
}

// device timeline of a completed request's unit in ms since the server was created (device clock):
// copies issued, host-to-device copies done, kernels started, kernels done; -1 where not (yet) known
extern "C" int b200_server_request_gpu_times(void *srv, int64_t id, double *times4)
{
    auto *s = (serve::Server *)srv;
    if (!s || !times4) return set_err(B200_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return set_err(B200_EINVAL, "unknown request id");
    const serve::Request *r = it->second;
    times4[0] = r->g_issued;
    times4[1] = r->g_copied;
    times4[2] = r->g_start;
    times4[3] = r->g_done;
    return B200_OK;
}

extern "C" int64_t b200_server_submit(void *srv, const uint64_t *host_trace, uint64_t nBits, uint64_t nBitsExt,
                                      uint64_t nCols, uint64_t arity, uint64_t *root_out)
{
    auto *s = (serve::Server *)srv;
    if (!s) return set_err(B200_EINVAL, "null server");
    int rc = check_shape(nBits, nBitsExt, nCols, arity);
    if (rc) return rc;
    if (nCols && !host_trace) return set_err(B200_EINVAL, "null trace");
    const int64_t id = s->submit(host_trace, (uint32_t)nBits, (uint32_t)nBitsExt, (uint32_t)nCols, (uint32_t)arity,
                                 root_out);
    if (id < 0) return set_err((int)id, "request larger than the device-memory budget");
    return id;
}

extern "C" int b200_server_status(void *srv, int64_t id, double *latency_ms)
{
    auto *s = (serve::Server *)srv;
    return s ? s->status(id, latency_ms) : set_err(B200_EINVAL, "null server");
}

extern "C" int b200_server_wait_all(void *srv, uint64_t timeout_ms)
{
    auto *s = (serve::Server *)srv;
    return s ? s->wait_all(timeout_ms) : set_err(B200_EINVAL, "null server");
}

extern "C" int b200_server_release(void *srv, int64_t id)
{
    auto *s = (serve::Server *)srv;
    return s ? s->release(id) : set_err(B200_EINVAL, "null server");
}

extern "C" int b200_server_buffers(void *srv, int64_t id, uint64_t **d_lde, uint64_t **d_tree)
{
    auto *s = (serve::Server *)srv;
    if (!s) return set_err(B200_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end() || it->second->status != 2 || it->second->released)
        return set_err(B200_EINVAL, "request not completed or released");
    if (d_lde) *d_lde = it->second->d_lde;
    if (d_tree) *d_tree = it->second->d_tree;
    return B200_OK;
}

extern "C" void b200_server_free(void *srv) { delete (serve::Server *)srv; }
