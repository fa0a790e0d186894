// Kernel-category timers and a launch counter (the reference's TimerGPU categories,
// utils/gpu_timer.cuh:15-276, as cudaEvent pairs recorded on the launching stream).
// Disabled by default; when enabled each category records one event pair per launch group.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <vector>

namespace prof {

enum Cat { TRANSPOSE = 0, NTT_INV, NTT_FWD, LEAF_HASH, TREE_LEVELS, NCAT };
static const char *const kCatNames[NCAT] = {"transpose", "ntt_inverse", "ntt_forward", "leaf_hash", "tree_levels"};

struct Pending {
    int cat;
    cudaEvent_t a, b;
};

static std::atomic<int> g_enabled{0};
static std::atomic<uint64_t> g_launches{0};
static std::mutex g_mu;
static std::vector<Pending> g_pending;
static double g_ms[NCAT];
static uint64_t g_count[NCAT];

inline void count(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

struct Scope {
    int cat;
    cudaStream_t s;
    cudaEvent_t a = nullptr, b = nullptr;
    Scope(int c, cudaStream_t st) : cat(c), s(st)
    {
        if (!g_enabled.load(std::memory_order_relaxed)) return;
        if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
            a = b = nullptr;
            return;
        }
        cudaEventRecord(a, s);
    }
    ~Scope()
    {
        if (!a) return;
        cudaEventRecord(b, s);
        std::lock_guard<std::mutex> lk(g_mu);
        g_pending.push_back(Pending{cat, a, b});
    }
};

// wait for recorded pairs and fold them into the per-category totals
inline void collect()
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto &p : g_pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            g_ms[p.cat] += ms;
            g_count[p.cat] += 1;
        }
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    g_pending.clear();
}

inline void reset()
{
    collect();
    std::lock_guard<std::mutex> lk(g_mu);
    for (int i = 0; i < NCAT; i++) {
        g_ms[i] = 0;
        g_count[i] = 0;
    }
}

}  // namespace prof
