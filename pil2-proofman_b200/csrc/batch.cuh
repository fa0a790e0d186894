// Batched commit of many AIR instances: grouped kernels and a persistent leaf-hash scheduler.
//
// The plain path runs each instance's kernel sequence on its own (transpose, NTT windows,
// leaf sponge, one launch per tree level).  Small instances then leave most of the GPU idle
// and every level of every tree is a separate launch.  Here one launch performs the same
// phase for every instance of the batch:
//   * grouped transpose, one launch per NTT window index (instances aligned on their last
//     inverse window and on their first forward window), one launch per tree level index;
//   * the leaf sponge is a persistent kernel: one resident CTA per SM slot pulls 128-row
//     blocks of any instance from a device work counter until all rows are hashed, so
//     instances of uneven size share the machine without tail effects;
// and the whole sequence is captured once in a CUDA graph and replayed (BatchPlan).
// Every kernel body is the plain path's body, so results are bit-identical to it.
#pragma once
#include <array>
#include <algorithm>
#include <cstring>
#include <vector>

#include "merkle.cuh"
#include "ntt.cuh"

namespace batch {

struct Inst {
    const uint64_t *trace;  // row-major N x nCols on the device
    uint64_t *scratch;      // N x nCols words
    uint64_t *lde;          // out: column-major NExt x nCols
    uint64_t *tree;         // out: tree_num_elements(NExt, arity) words
    uint32_t nBits, nBitsExt, nCols, arity;
};

struct TransposeEntry {
    const uint64_t *src;
    uint64_t *dst;
    uint64_t nrows, ncols, rtiles, ctiles, begin;
};

struct PassEntry {
    ntt::Pass p;
    uint64_t tiles, ncols, begin;
};

struct LeafEntry {
    const uint64_t *src;
    uint64_t *digests;
    uint64_t ncols, nrows, begin;  // begin: first 128-row block index of this entry
};

struct NodeEntry {
    uint64_t *level, *out;
    uint64_t pending, pad, parents, begin;
};

// index of the entry owning global block b (entries sorted by begin, begin[0] = 0)
template <typename E>
__device__ __forceinline__ int find_entry(const E *e, int n, uint64_t b)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (e[mid].begin <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(256) transpose_grouped(const TransposeEntry *e, int n)
{
    const int i = find_entry(e, n, blockIdx.x);
    const TransposeEntry t = e[i];
    const uint64_t local = blockIdx.x - t.begin;
    ntt::transpose_tile(t.dst, t.src, t.nrows, t.ncols, t.nrows, local % t.rtiles, local / t.rtiles);
}

__global__ void __launch_bounds__(512, 2) pass_grouped(const PassEntry *e, int n)
{
    __shared__ ntt::Pass p;  // staged like pass_fixed_grouped's
    __shared__ uint32_t tile, col;
    if (threadIdx.x == 0) {
        const int i = find_entry(e, n, blockIdx.x);
        p = e[i].p;
        const uint32_t local = (uint32_t)(blockIdx.x - e[i].begin), tiles = (uint32_t)e[i].tiles;
        tile = local % tiles;
        col = local / tiles;
    }
    __syncthreads();
    ntt::pass16_body(p, tile, col);
}

// Grouped fixed-shape window: every entry of the launch has window shape (K, LGL) and
// direction DIF.
template <int K, int LGL, bool DIF>
__global__ void __launch_bounds__(ntt::Shape<K, LGL>::NT, 1024 / ntt::Shape<K, LGL>::NT)
    pass_fixed_grouped(const PassEntry *e, int n)
{
    // the entry's window description staged in shared memory (read there as needed, not held in
    // registers: a register copy of the struct pushed the window bodies into spills)
    __shared__ ntt::Pass p;
    __shared__ uint32_t tile, col;
    if (threadIdx.x == 0) {
        const int i = find_entry(e, n, blockIdx.x);
        p = e[i].p;
        // block and tile counts of a launch are below 2^31
        const uint32_t local = (uint32_t)(blockIdx.x - e[i].begin), tiles = (uint32_t)e[i].tiles;
        tile = local % tiles;
        col = local / tiles;
    }
    __syncthreads();
    ntt::pass_fixed_body<K, LGL, DIF>(p, tile, col);
}

typedef void (*GroupedKernel)(const PassEntry *, int);

template <int K>
inline GroupedKernel grouped_fixed_k(uint32_t lgL, uint32_t dif)
{
    if (lgL == 13 - K) return dif ? pass_fixed_grouped<K, 13 - K, true> : pass_fixed_grouped<K, 13 - K, false>;
    if (lgL == 0) return dif ? pass_fixed_grouped<K, 0, true> : pass_fixed_grouped<K, 0, false>;
    return nullptr;
}

// the grouped fixed-shape kernel of a window shape and direction, or null (the generic grouped
// kernel serves it)
inline GroupedKernel grouped_fixed(uint32_t k, uint32_t lgL, uint32_t dif)
{
    switch (k) {
    case 1: return grouped_fixed_k<1>(lgL, dif);
    case 2: return grouped_fixed_k<2>(lgL, dif);
    case 3: return grouped_fixed_k<3>(lgL, dif);
    case 4: return grouped_fixed_k<4>(lgL, dif);
    case 5: return grouped_fixed_k<5>(lgL, dif);
    case 6: return grouped_fixed_k<6>(lgL, dif);
    case 7: return grouped_fixed_k<7>(lgL, dif);
    case 8: return grouped_fixed_k<8>(lgL, dif);
    case 9: return grouped_fixed_k<9>(lgL, dif);
    case 10: return grouped_fixed_k<10>(lgL, dif);
    case 11: return grouped_fixed_k<11>(lgL, dif);
    case 12: return grouped_fixed_k<12>(lgL, dif);
    default: return nullptr;
    }
}

inline cudaError_t set_grouped_fixed_attrs()
{
    for (uint32_t k = 1; k <= NTT_KMAX; k++) {
        const uint32_t shapes[2] = {13 - k, 0};
        for (uint32_t lgL : shapes)
            for (uint32_t dif = 0; dif < 2; dif++) {
                GroupedKernel g = grouped_fixed(k, lgL, dif);
                if (!g) continue;
                const uint32_t T = 1u << (k + lgL);
                cudaError_t e =
                    cudaFuncSetAttribute(g, cudaFuncAttributeMaxDynamicSharedMemorySize, (T + T / 16) * 8);
                if (e != cudaSuccess) return e;
            }
    }
    return cudaSuccess;
}

// Persistent leaf sponge: CTAs claim 128-row blocks from *counter until `total` is reached.
template <int W, int FAM>
__global__ void __launch_bounds__(merkle::TPB, merkle::Family<FAM>::MIN_CTAS)
    leaf_persistent(const LeafEntry *e, int n, uint64_t total, unsigned long long *counter)
{
    __shared__ uint64_t sm[merkle::Family<FAM>::SMEM_AREAS * W * merkle::TPB];
    __shared__ uint64_t claim;
    __shared__ LeafEntry L;  // the claimed block's instance, staged for the CTA
    for (;;) {
        if (threadIdx.x == 0) {
            claim = atomicAdd(counter, 1ull);
            if (claim < total) L = e[find_entry(e, n, claim)];
        }
        __syncthreads();
        const uint64_t b = claim;
        if (b >= total) return;
        const uint64_t row = (b - L.begin) * merkle::TPB + threadIdx.x;
        if (row < L.nrows) merkle::leaf_row<W, FAM>(sm + threadIdx.x, L.digests, L.src, 1, L.nrows, L.ncols, row);
        __syncthreads();
    }
}

template <int W, int FAM>
__global__ void __launch_bounds__(merkle::TPB, merkle::Family<FAM>::MIN_CTAS) node_grouped(const NodeEntry *e, int n)
{
    __shared__ uint64_t sm[merkle::Family<FAM>::SMEM_AREAS * W * merkle::TPB];
    const int i = find_entry(e, n, blockIdx.x);
    const NodeEntry E = e[i];
    const uint64_t idx = (blockIdx.x - E.begin) * merkle::TPB + threadIdx.x;
    if (idx < E.parents) merkle::node_one<W, FAM>(sm + threadIdx.x, E.level, E.pending, E.pad, E.parents, E.out, idx);
}

__global__ void gather_roots(const uint64_t *const *tree_ends, int n, uint64_t *roots)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 4 * n) roots[i] = tree_ends[i >> 2][i & 3];
}

// ------------------------------------------------------------------ host plan ----

// Instances whose window (or transpose) covers at least this many elements get the plain path's
// own launch for it: such a launch alone fills the GPU for dozens of waves, and the plain kernel
// reads its window description from the kernel parameters, where the grouped kernel first finds
// its entry and stages it through shared memory (measured on B200: grouped windows 2-8 % and the
// grouped transpose 14 % slower than the plain launches of the same instances).
constexpr uint64_t PLAIN_MIN_ELEMS = 1ull << 27;

struct Launch {
    // 0 transpose, 1 pass (generic), 2 leaf, 3 node, 5 pass (fixed shape width, lgl, dif),
    // 6 one instance's window as a plain launch, 7 one instance's transpose as a plain launch
    int kind;
    int width;
    size_t off;  // byte offset of the entry array in the device table buffer
    int n;
    uint64_t blocks;
    size_t smem;
    int lgl = 0;
    int dif = 0;
    ntt::Pass pass{};   // kind 6
    uint64_t ncols = 0; // kind 6
    int inst = -1;      // kind 7
};

class Plan {
  public:
    std::vector<Inst> inst;
    std::vector<Launch> launches;
    std::vector<unsigned char> table;  // host image of the device table buffer
    unsigned char *d_table = nullptr;
    size_t counters_off = 0, roots_off = 0, ends_off = 0;
    int n_counters = 0;
    uint64_t *h_roots = nullptr;  // pinned, 4 words per instance
    cudaGraphExec_t graph = nullptr;
    int leaf_ctas = 0;
    int family = 2;  // hash family of the leaves and levels (1 = Poseidon1, 2 = Poseidon2)
    // d_table and h_roots belong to the caller (the commit server's pool and pinned staging)
    bool borrowed = false;

    ~Plan() { release(); }

    void release()
    {
        if (graph) cudaGraphExecDestroy(graph);
        if (d_table && !borrowed) cudaFree(d_table);
        if (h_roots && !borrowed) cudaFreeHost(h_roots);
        graph = nullptr;
        d_table = nullptr;
        h_roots = nullptr;
    }

    // one window index's entries as launches: one per fixed window shape and direction, the
    // rest generic
    void push_passes(const std::vector<PassEntry> &all)
    {
        std::vector<PassEntry> pe;
        for (const PassEntry &e : all) {
            if ((e.tiles << (e.p.k + e.p.lgL)) * e.ncols >= PLAIN_MIN_ELEMS) {
                Launch L{6, 0, 0, 1, e.tiles * e.ncols, 0};
                L.pass = e.p;
                L.ncols = e.ncols;
                launches.push_back(L);
            } else {
                pe.push_back(e);
            }
        }
        std::vector<std::array<uint32_t, 3>> shapes;
        for (const PassEntry &e : pe) {
            const std::array<uint32_t, 3> sh{e.p.k, e.p.lgL, e.p.dif ? 1u : 0u};
            if (grouped_fixed(sh[0], sh[1], sh[2]) && std::find(shapes.begin(), shapes.end(), sh) == shapes.end())
                shapes.push_back(sh);
        }
        for (const auto &sh : shapes) {
            std::vector<PassEntry> g;
            uint64_t b = 0;
            for (PassEntry e : pe)
                if (e.p.k == sh[0] && e.p.lgL == sh[1] && (e.p.dif ? 1u : 0u) == sh[2]) {
                    e.begin = b;
                    b += e.tiles * e.ncols;
                    g.push_back(e);
                }
            const size_t T = 1ull << (sh[0] + sh[1]);
            Launch L{5, (int)sh[0], push(g), (int)g.size(), b, (T + T / 16) * 8};
            L.lgl = (int)sh[1];
            L.dif = (int)sh[2];
            launches.push_back(L);
        }
        std::vector<PassEntry> rest;
        uint64_t b = 0;
        size_t smem = 0;
        for (PassEntry e : pe)
            if (!grouped_fixed(e.p.k, e.p.lgL, e.p.dif)) {
                e.begin = b;
                b += e.tiles * e.ncols;
                const size_t T = 1ull << (e.p.k + e.p.lgL);
                smem = std::max(smem, (T + T / 16) * 8);
                rest.push_back(e);
            }
        if (!rest.empty()) launches.push_back(Launch{1, 0, push(rest), (int)rest.size(), b, smem});
    }

    template <typename T>
    size_t push(const std::vector<T> &v)
    {
        size_t off = (table.size() + 255) & ~size_t(255);
        table.resize(off + v.size() * sizeof(T));
        if (!v.empty()) memcpy(table.data() + off, v.data(), v.size() * sizeof(T));
        return off;
    }

    // Builds the launch list for `in`; returns false on an unsupported shape.
    bool build(const std::vector<Inst> &in, int sm_count, int fam = 2)
    {
        inst = in;
        family = fam == 1 ? 1 : 2;
        launches.clear();
        table.clear();
        // transpose
        {
            std::vector<TransposeEntry> te;
            uint64_t b = 0;
            for (size_t i = 0; i < inst.size(); i++) {
                const Inst &x = inst[i];
                const uint64_t N = 1ull << x.nBits;
                if (!x.nCols) continue;
                if (N * x.nCols >= PLAIN_MIN_ELEMS) {
                    Launch L{7, 0, 0, 1, 0, 0};
                    L.inst = (int)i;
                    launches.push_back(L);
                    continue;
                }
                TransposeEntry t{x.trace, x.scratch, N, x.nCols, (N + 31) / 32, (x.nCols + 31) / 32ull, b};
                b += t.rtiles * t.ctiles;
                te.push_back(t);
            }
            if (!te.empty()) launches.push_back(Launch{0, 0, push(te), (int)te.size(), b, 0});
        }
        // inverse windows, aligned on the last (coset-scaling) window
        std::vector<std::vector<ntt::Window>> dif(inst.size()), dit(inst.size());
        int maxd = 0, maxf = 0;
        for (size_t i = 0; i < inst.size(); i++) {
            ntt::Window w[8];
            const Inst &x = inst[i];
            const ntt::Tune tn = ntt::tuned(x.nBits, x.nBitsExt, x.nCols);
            int nw = x.nBits ? ntt::plan_windows(0, x.nBits, w, 8, tn.kfirst, tn.krest) : 0;
            if (nw < 0) return false;
            dif[i].assign(w, w + nw);
            nw = ntt::plan_windows(x.nBitsExt - x.nBits, x.nBitsExt, w, 8, tn.kfirst, tn.krest);
            if (nw < 0) return false;
            dit[i].assign(w, w + nw);
            maxd = std::max(maxd, (int)dif[i].size());
            maxf = std::max(maxf, (int)dit[i].size());
        }
        for (int j = maxd - 1; j >= 0; j--) {
            std::vector<PassEntry> pe;
            uint64_t b = 0;
            size_t smem = 0;
            for (size_t i = 0; i < inst.size(); i++) {
                const Inst &x = inst[i];
                if (j >= (int)dif[i].size() || !x.nCols) continue;
                const ntt::Window &w = dif[i][j];
                const uint64_t N = 1ull << x.nBits;
                PassEntry e{};
                e.p.src = x.scratch;
                e.p.dst = x.scratch;
                e.p.src_cs = N;
                e.p.dst_cs = N;
                e.p.lg = x.nBits;
                e.p.s0 = w.s0;
                e.p.k = w.k;
                e.p.lgL = w.lgL;
                e.p.rep = 0;
                e.p.dif = 1;
                e.p.post = (j == 0) ? ntt::POST_COSET : ntt::POST_NONE;
                e.tiles = N >> (w.k + w.lgL);
                e.ncols = x.nCols;
                e.begin = b;
                b += e.tiles * e.ncols;
                const size_t T = 1ull << (w.k + w.lgL);
                smem = std::max(smem, (T + T / 16) * 8);
                pe.push_back(e);
            }
            (void)smem;
            if (!pe.empty()) push_passes(pe);
        }
        for (int j = 0; j < maxf; j++) {
            std::vector<PassEntry> pe;
            uint64_t b = 0;
            size_t smem = 0;
            for (size_t i = 0; i < inst.size(); i++) {
                const Inst &x = inst[i];
                if (j >= (int)dit[i].size() || !x.nCols) continue;
                const ntt::Window &w = dit[i][j];
                const uint64_t N = 1ull << x.nBits, NExt = 1ull << x.nBitsExt;
                PassEntry e{};
                e.p.src = (j == 0) ? (const uint64_t *)x.scratch : x.lde;
                e.p.dst = x.lde;
                e.p.src_cs = (j == 0) ? N : NExt;
                e.p.dst_cs = NExt;
                e.p.lg = x.nBitsExt;
                e.p.s0 = w.s0;
                e.p.k = w.k;
                e.p.lgL = w.lgL;
                e.p.rep = (j == 0) ? (x.nBitsExt - x.nBits) : 0;
                e.p.dif = 0;
                e.p.post = (j == (int)dit[i].size() - 1) ? ntt::POST_CANON : ntt::POST_NONE;
                e.tiles = NExt >> (w.k + w.lgL);
                e.ncols = x.nCols;
                e.begin = b;
                b += e.tiles * e.ncols;
                const size_t T = 1ull << (w.k + w.lgL);
                smem = std::max(smem, (T + T / 16) * 8);
                pe.push_back(e);
            }
            (void)smem;
            if (!pe.empty()) push_passes(pe);
        }
        // leaves (one persistent launch per arity) and tree levels
        n_counters = 0;
        std::vector<size_t> counter_slots;
        for (uint32_t ar = 2; ar <= 4; ar++) {
            std::vector<LeafEntry> le;
            uint64_t b = 0;
            for (const Inst &x : inst) {
                if (x.arity != ar) continue;
                const uint64_t NExt = 1ull << x.nBitsExt;
                LeafEntry e{x.lde, x.tree, x.nCols, NExt, b};
                b += (NExt + merkle::TPB - 1) / merkle::TPB;
                le.push_back(e);
            }
            if (le.empty()) continue;
            Launch L{2, (int)(4 * ar), push(le), (int)le.size(), b, 0};
            L.smem = (size_t)n_counters++;  // counter index
            launches.push_back(L);
            // levels
            for (int lvl = 0;; lvl++) {
                std::vector<NodeEntry> ne;
                uint64_t nb = 0;
                for (const Inst &x : inst) {
                    if (x.arity != ar) continue;
                    uint64_t pending = 1ull << x.nBitsExt, base = 0;
                    int l = 0;
                    while (pending > 1 && l < lvl) {
                        const uint64_t pad = (ar - pending % ar) % ar;
                        base += (pending + pad) * 4;
                        pending = (pending + ar - 1) / ar;
                        l++;
                    }
                    if (pending <= 1) continue;
                    const uint64_t pad = (ar - pending % ar) % ar, parents = (pending + ar - 1) / ar;
                    NodeEntry e{x.tree + base, x.tree + base + (pending + pad) * 4, pending, pad, parents, nb};
                    nb += (parents + merkle::TPB - 1) / merkle::TPB;
                    ne.push_back(e);
                }
                if (ne.empty()) break;
                launches.push_back(Launch{3, (int)(4 * ar), push(ne), (int)ne.size(), nb, 0});
            }
        }
        // roots: pointers to the last 4 words of every tree
        std::vector<const uint64_t *> ends;
        for (const Inst &x : inst)
            ends.push_back(x.tree + merkle::tree_num_elements(1ull << x.nBitsExt, x.arity) - 4);
        ends_off = push(ends);
        std::vector<uint64_t> zeros(4 * inst.size() + 1, 0);
        roots_off = push(zeros);
        std::vector<unsigned long long> ctr(n_counters ? n_counters : 1, 0ull);
        counters_off = push(ctr);
        leaf_ctas = sm_count * merkle::Family<2>::MIN_CTAS;
        if (family == 1) leaf_ctas = sm_count * merkle::Family<1>::MIN_CTAS;
        return true;
    }

    // device copy of the descriptor tables and a pinned root buffer (once per plan)
    cudaError_t upload()
    {
        if (d_table) return cudaSuccess;
        cudaError_t e = cudaMalloc((void **)&d_table, table.size());
        if (e != cudaSuccess) return e;
        e = cudaMemcpy(d_table, table.data(), table.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return e;
        return cudaMallocHost((void **)&h_roots, 32 * (inst.size() + 1));
    }

    // the whole batch: grouped launches, persistent leaves, levels, roots -> h_roots
    cudaError_t enqueue(cudaStream_t s)
    {
        cudaError_t e;
        unsigned long long *ctr = (unsigned long long *)(d_table + counters_off);
        if (n_counters && (e = cudaMemsetAsync(ctr, 0, 8 * n_counters, s)) != cudaSuccess) return e;
        for (const Launch &L : launches) {
            const void *ent = d_table + L.off;
            switch (L.kind) {
            case 0: transpose_grouped<<<(unsigned)L.blocks, dim3(32, 8), 0, s>>>((const TransposeEntry *)ent, L.n); break;
            case 6:
                if ((e = ntt::launch_pass(L.pass, L.ncols, s)) != cudaSuccess) return e;
                continue;  // launch_pass counts its launch
            case 7: {
                const Inst &x = inst[(size_t)L.inst];
                const uint64_t N = 1ull << x.nBits;
                if ((e = ntt::transpose(x.scratch, x.trace, N, x.nCols, N, s)) != cudaSuccess) return e;
                continue;  // transpose counts its launch
            }
            case 1: pass_grouped<<<(unsigned)L.blocks, 512, L.smem, s>>>((const PassEntry *)ent, L.n); break;
            case 5: {
                const uint32_t T = 1u << (L.width + L.lgl);
                const uint32_t nt = T / 16 < 32 ? 32 : T / 16 > 512 ? 512 : T / 16;
                grouped_fixed((uint32_t)L.width, (uint32_t)L.lgl, (uint32_t)L.dif)<<<(unsigned)L.blocks, nt, L.smem, s>>>(
                    (const PassEntry *)ent, L.n);
                break;
            }
            case 2: {
                const unsigned ctas = (unsigned)std::min<uint64_t>(L.blocks, (uint64_t)leaf_ctas);
                const LeafEntry *le = (const LeafEntry *)ent;
                if (family == 1) {
                    if (L.width == 8) leaf_persistent<8, 1><<<ctas, merkle::TPB, 0, s>>>(le, L.n, L.blocks, ctr + L.smem);
                    if (L.width == 12) leaf_persistent<12, 1><<<ctas, merkle::TPB, 0, s>>>(le, L.n, L.blocks, ctr + L.smem);
                    if (L.width == 16) leaf_persistent<16, 1><<<ctas, merkle::TPB, 0, s>>>(le, L.n, L.blocks, ctr + L.smem);
                } else {
                    if (L.width == 8) leaf_persistent<8, 2><<<ctas, merkle::TPB, 0, s>>>(le, L.n, L.blocks, ctr + L.smem);
                    if (L.width == 12) leaf_persistent<12, 2><<<ctas, merkle::TPB, 0, s>>>(le, L.n, L.blocks, ctr + L.smem);
                    if (L.width == 16) leaf_persistent<16, 2><<<ctas, merkle::TPB, 0, s>>>(le, L.n, L.blocks, ctr + L.smem);
                }
                break;
            }
            case 3: {
                const NodeEntry *ne = (const NodeEntry *)ent;
                if (family == 1) {
                    if (L.width == 8) node_grouped<8, 1><<<(unsigned)L.blocks, merkle::TPB, 0, s>>>(ne, L.n);
                    if (L.width == 12) node_grouped<12, 1><<<(unsigned)L.blocks, merkle::TPB, 0, s>>>(ne, L.n);
                    if (L.width == 16) node_grouped<16, 1><<<(unsigned)L.blocks, merkle::TPB, 0, s>>>(ne, L.n);
                } else {
                    if (L.width == 8) node_grouped<8, 2><<<(unsigned)L.blocks, merkle::TPB, 0, s>>>(ne, L.n);
                    if (L.width == 12) node_grouped<12, 2><<<(unsigned)L.blocks, merkle::TPB, 0, s>>>(ne, L.n);
                    if (L.width == 16) node_grouped<16, 2><<<(unsigned)L.blocks, merkle::TPB, 0, s>>>(ne, L.n);
                }
                break;
            }
            }
            prof::count();
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        uint64_t *d_roots = (uint64_t *)(d_table + roots_off);
        const int n = (int)inst.size();
        gather_roots<<<(4 * n + 127) / 128, 128, 0, s>>>((const uint64_t *const *)(d_table + ends_off), n, d_roots);
        prof::count();
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        return cudaMemcpyAsync(h_roots, d_roots, 32 * n, cudaMemcpyDeviceToHost, s);
    }

    // Runs the batch on `s` (a created stream, not the legacy default stream, when use_graph):
    // the first graph run captures the launch sequence once; later runs replay it.
    cudaError_t run(cudaStream_t s, bool use_graph)
    {
        cudaError_t e = upload();
        if (e != cudaSuccess) return e;
        if (!use_graph) return enqueue(s);
        if (!graph) {
            cudaGraph_t g;
            if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
            cudaError_t qe = enqueue(s);
            e = cudaStreamEndCapture(s, &g);
            if (qe != cudaSuccess) return qe;
            if (e != cudaSuccess) return e;
            e = cudaGraphInstantiate(&graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return e;
        }
        return cudaGraphLaunch(graph, s);
    }
};

}  // namespace batch
