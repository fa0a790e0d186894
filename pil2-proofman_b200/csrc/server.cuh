// Commit server: a request loop with continuous admission (included at the end of pil2_b200.cu).
//
// Requests (host row-major traces) arrive at any time.  A worker thread admits them in arrival
// order whenever a stream slot is free and the device-memory budget holds the request's buffers
// (trace, scratch, LDE, tree); each admitted request runs H2D -> LDE -> tree -> root D2H on its own
// stream, so requests admitted while others are on the GPU overlap with them.  Completion is
// observed through an event; the LDE and the tree stay resident on the device (for later query
// reads) until the caller releases the request.  Device buffers come from the stream-ordered pool
// (cudaMallocAsync), which keeps freed memory cached for the next admissions.  No call blocks on
// the GPU except b200_server_wait_all, whose wait is bounded by its timeout.
#pragma once
#include <chrono>
#include <condition_variable>
#include <deque>
#include <unordered_map>

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
    uint64_t *h_root = nullptr;  // pinned 4 words
    cudaEvent_t done = nullptr;
    int slot = -1;
    int status = 0;  // 0 queued, 1 running, 2 done, < 0 error
    bool released = false;
    double t_submit = 0, t_admit = 0, t_done = 0;
    std::string err;  // reason of a failed request (reported to the caller by status())
    uint64_t bytes() const { return 8 * (2 * words_trace + words_lde + words_tree); }
};

class Server {
  public:
    int device = 0;
    uint64_t budget = 0, used = 0;
    std::vector<cudaStream_t> streams;
    std::vector<int> slot_busy;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request *> queue;
    std::vector<Request *> running;
    std::unordered_map<int64_t, Request *> all;
    int64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    cudaMemPool_t pool = nullptr;
    cudaEvent_t last_done = nullptr;  // completion event of the most recently admitted request
    int family = 2;                   // hash family of this server's commits (fixed at creation)

    int start(int dev, uint64_t budget_bytes, uint32_t slots)
    {
        device = dev;
        budget = budget_bytes;
        CK(cudaSetDevice(dev), "cudaSetDevice");
        int rc = ensure_init_current();
        if (rc) return rc;
        CK(cudaDeviceGetDefaultMemPool(&pool, dev), "mem pool");
        uint64_t keep = UINT64_MAX;  // keep freed blocks cached in the pool
        CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "mem pool threshold");
        for (uint32_t i = 0; i < slots; i++) {
            cudaStream_t s;
            CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
            streams.push_back(s);
            slot_busy.push_back(0);
        }
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
        for (auto &kv : all) {
            Request *r = kv.second;
            if (r->done) cudaEventSynchronize(r->done);
            free_buffers(r, nullptr);
            if (r->done) cudaEventDestroy(r->done);
            if (r->h_root) cudaFreeHost(r->h_root);
            delete r;
        }
        for (cudaStream_t s : streams) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }

    void free_buffers(Request *r, cudaStream_t s)
    {
        for (uint64_t **p : {&r->d_trace, &r->d_scratch, &r->d_lde, &r->d_tree})
            if (*p) {
                cudaFreeAsync(*p, s);
                *p = nullptr;
            }
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
        }
        cv.notify_all();
        return r->id;
    }

    // all four device buffers of a request, or none
    bool alloc_request(Request *r, cudaStream_t s)
    {
        if (cudaMallocAsync((void **)&r->d_trace, 8 * (r->words_trace ? r->words_trace : 1), s) == cudaSuccess &&
            cudaMallocAsync((void **)&r->d_scratch, 8 * (r->words_trace ? r->words_trace : 1), s) == cudaSuccess &&
            cudaMallocAsync((void **)&r->d_lde, 8 * (r->words_lde ? r->words_lde : 1), s) == cudaSuccess &&
            cudaMallocAsync((void **)&r->d_tree, 8 * r->words_tree, s) == cudaSuccess)
            return true;
        cudaGetLastError();
        free_buffers(r, s);
        return false;
    }

    // admit the head of the queue onto a free slot; caller holds mu
    bool admit_one()
    {
        if (queue.empty()) return false;
        Request *r = queue.front();
        int slot = -1;
        for (size_t i = 0; i < streams.size(); i++)
            if (!slot_busy[i]) {
                slot = (int)i;
                break;
            }
        if (slot < 0 || used + r->bytes() > budget) return false;
        queue.pop_front();
        cudaStream_t s = streams[slot];
        r->slot = slot;
        r->t_admit = now_ms();
        int rc = B200_OK;
        if (!r->h_root && cudaMallocHost((void **)&r->h_root, 32) != cudaSuccess) rc = B200_ENOMEM;
        if (!rc && !r->done && cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming) != cudaSuccess)
            rc = B200_ECUDA;
        if (!rc && !alloc_request(r, s)) {
            // The pool keeps freed blocks cached; when the cached sizes do not fit this request,
            // return them to the device (after the running requests' frees have executed) and retry.
            for (cudaStream_t t : streams) cudaStreamSynchronize(t);
            cudaMemPoolTrimTo(pool, 0);
            cudaGetLastError();
            if (!alloc_request(r, s)) {
                rc = B200_ENOMEM;
                r->err = "device buffers for the request could not be allocated";
            }
        }
        if (!rc && r->words_trace &&
            cudaMemcpyAsync(r->d_trace, r->trace, 8 * r->words_trace, cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = B200_ECUDA;
        // kernels of admitted requests run in admission order (the H2D above overlaps the previous
        // request's kernels); interleaved requests would each take longer and finish together
        if (!rc && last_done) cudaStreamWaitEvent(s, last_done, 0);
        if (!rc) rc = commit_device_fam(nullptr, r->d_lde, r->d_tree, r->d_trace, 1, r->nBits, r->nBitsExt, r->nCols,
                                        r->arity, r->d_scratch, s, family);
        if (!rc && cudaMemcpyAsync(r->h_root, r->d_tree + r->words_tree - 4, 32, cudaMemcpyDeviceToHost, s) !=
                       cudaSuccess)
            rc = B200_ECUDA;
        if (!rc) {
            // the trace copy and the scratch are not needed once the commit has run
            cudaFreeAsync(r->d_trace, s);
            cudaFreeAsync(r->d_scratch, s);
            r->d_trace = r->d_scratch = nullptr;
            if (cudaEventRecord(r->done, s) != cudaSuccess) rc = B200_ECUDA;
            else last_done = r->done;
        }
        if (rc) {
            free_buffers(r, s);
            if (r->err.empty()) r->err = "request failed on the device (CUDA error)";
            r->status = rc;
            r->t_done = now_ms();
            return true;
        }
        used += r->bytes();
        slot_busy[slot] = 1;
        r->status = 1;
        running.push_back(r);
        return true;
    }

    // caller holds mu
    void harvest()
    {
        for (size_t i = 0; i < running.size();) {
            Request *r = running[i];
            if (cudaEventQuery(r->done) == cudaSuccess) {
                r->t_done = now_ms();
                if (r->root_out) memcpy(r->root_out, r->h_root, 32);
                r->status = 2;
                slot_busy[r->slot] = 0;
                used -= 8 * 2 * r->words_trace;  // trace + scratch were freed at admission
                running[i] = running.back();
                running.pop_back();
            } else {
                i++;
            }
        }
    }

    void loop()
    {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lk(mu);
        while (!stop) {
            harvest();
            while (admit_one()) {
            }
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
            free_buffers(r, streams[r->slot >= 0 ? r->slot : 0]);
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
