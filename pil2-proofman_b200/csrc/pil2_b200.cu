// pil2_b200: the commit path (LDE + Poseidon2 Merkle) behind the reference's C ABI.
// One translation unit: the kernels (ntt.cuh, merkle.cuh) share __constant__/__device__
// tables with the drivers below.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/pil2_b200.h"
#include "merkle.cuh"
#include "ntt.cuh"
#include "stark_info.cuh"
#include "stream.cuh"
#include "synth.cuh"

// ------------------------------------------------------------------ errors ----
static thread_local std::string t_err;
static int set_err(int code, const std::string &msg)
{
    t_err = msg;
    return code;
}
static int cuda_err(cudaError_t e, const char *where)
{
    return set_err(B200_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define CK(call, where)                                  \
    do {                                                 \
        cudaError_t _e = (call);                         \
        if (_e != cudaSuccess) return cuda_err(_e, where); \
    } while (0)

extern "C" const char *b200_last_error(void) { return t_err.c_str(); }

// ------------------------------------------------------------- per device ----
static std::mutex g_init_mu;
static bool g_init_done[64];

static int ensure_init_current()
{
    int dev = 0;
    CK(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) return set_err(B200_EINVAL, "device index out of range");
    std::lock_guard<std::mutex> lk(g_init_mu);
    if (g_init_done[dev]) return B200_OK;
    CK(ntt::init_tables(), "ntt tables");
    CK(cudaFuncSetAttribute(ntt::pass16_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (NTT_TILE_MAX + NTT_TILE_MAX / 16) * 8),
       "pass16_kernel smem attribute");
    CK(ntt::set_fixed_attrs(), "pass_fixed_kernel smem attributes");
    g_init_done[dev] = true;
    return B200_OK;
}

extern "C" int b200_init(int device)
{
    CK(cudaSetDevice(device), "cudaSetDevice");
    return ensure_init_current();
}

extern "C" int b200_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

extern "C" uint64_t b200_tree_num_elements(uint64_t nrows, uint64_t arity)
{
    if (arity < 2) return 0;
    return merkle::tree_num_elements(nrows, arity);
}

extern "C" uint64_t b200_lde_scratch_words(uint64_t nBits, uint64_t nCols)
{
    return ntt::lde_scratch_words((uint32_t)nBits, nCols);
}

static int check_shape(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t arity)
{
    if (nBitsExt < nBits) return set_err(B200_EINVAL, "nBitsExt < nBits");
    if (nBitsExt > NTT_TWLG) return set_err(B200_EINVAL, "nBitsExt above 26");
    if (nBitsExt - nBits > 12) return set_err(B200_EINVAL, "blowup above 2^12");
    if (nCols > 65535) return set_err(B200_EINVAL, "nCols above 65535");
    if (arity < 2 || arity > 4) return set_err(B200_EINVAL, "arity must be 2, 3 or 4");
    return B200_OK;
}

// Hash family of the native b200_* entry points (1 = Poseidon1, 2 = Poseidon2, the default).
// The reference entry points follow set_hash_family instead, which the reference allows to be
// set once per process.
static std::atomic<int> g_native_family{2};

extern "C" int b200_set_native_hash_family(int family)
{
    if (family != 1 && family != 2) return set_err(B200_EINVAL, "hash family must be 1 (Poseidon1) or 2 (Poseidon2)");
    g_native_family.store(family);
    return B200_OK;
}

extern "C" int b200_native_hash_family(void) { return g_native_family.load(); }

// ------------------------------------------------------- device-pointer API ----
extern "C" int b200_lde_device(uint64_t *d_lde, const uint64_t *d_trace, int trace_rowmajor, uint64_t nBits,
                               uint64_t nBitsExt, uint64_t nCols, uint64_t *d_scratch, void *stream)
{
    int rc = check_shape(nBits, nBitsExt, nCols, 4);
    if (rc) return rc;
    if ((rc = ensure_init_current())) return rc;
    if (nCols && (!d_lde || !d_trace || !d_scratch)) return set_err(B200_EINVAL, "null buffer");
    CK(ntt::lde(d_lde, d_trace, trace_rowmajor != 0, (uint32_t)nBits, (uint32_t)nBitsExt, nCols, d_scratch,
                (cudaStream_t)stream),
       "lde");
    return B200_OK;
}

// ---------------------------------------- LDE with the library's own scratch area ----
// Some callers may not allocate device memory at all: a prover that hands the library only
// buffers carved from its own pool (torch's caching allocator, a preallocated arena under a
// fixed memory budget), or a latency-critical loop that cannot afford cudaMalloc's implicit
// device synchronisation.  For them the LDE runs with a scratch area that is part of this
// library's image: a file-scope device array, loaded with the module and held by every GPU
// that loads the library until the process exits.
#define B200_STATIC_SCRATCH_WORDS (1ull << 23)  // 64 MiB: N * nCols <= 2^23 words
static __device__ __align__(256) uint64_t g_static_lde_scratch[B200_STATIC_SCRATCH_WORDS];
static uint64_t *g_static_scratch_addr[64];  // device address of the array, per device
static std::mutex g_static_scratch_mu;

extern "C" int b200_lde_device_static_scratch(uint64_t *d_lde, const uint64_t *d_trace, int trace_rowmajor,
                                              uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, void *stream)
{
    int rc = check_shape(nBits, nBitsExt, nCols, 4);
    if (rc) return rc;
    const uint64_t words = ntt::lde_scratch_words((uint32_t)nBits, nCols);
    if (words > B200_STATIC_SCRATCH_WORDS)
        return set_err(B200_EINVAL, "b200_lde_device_static_scratch: needs " + std::to_string(words) +
                                        " scratch words, the built-in area holds " +
                                        std::to_string(B200_STATIC_SCRATCH_WORDS) + " (N * nCols <= 2^23)");
    if (nCols && (!d_lde || !d_trace)) return set_err(B200_EINVAL, "null buffer");
    if ((rc = ensure_init_current())) return rc;
    int dev = 0;
    CK(cudaGetDevice(&dev), "cudaGetDevice");
    uint64_t *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_static_scratch_mu);
        if (!g_static_scratch_addr[dev]) {
            // the array's name is a host-side stand-in; the kernels need its device address
            void *p = nullptr;
            CK(cudaGetSymbolAddress(&p, g_static_lde_scratch), "cudaGetSymbolAddress(static LDE scratch)");
            g_static_scratch_addr[dev] = (uint64_t *)p;
        }
        scratch = g_static_scratch_addr[dev];
    }
    CK(ntt::lde(d_lde, d_trace, trace_rowmajor != 0, (uint32_t)nBits, (uint32_t)nBitsExt, nCols, scratch,
                (cudaStream_t)stream),
       "lde (static scratch)");
    return B200_OK;
}

extern "C" int b200_merkletree_device(uint64_t *d_tree, const uint64_t *d_src, uint64_t rs, uint64_t cs,
                                      uint64_t nCols, uint64_t nRows, uint64_t arity, void *stream)
{
    if (arity < 2 || arity > 4) return set_err(B200_EINVAL, "arity must be 2, 3 or 4");
    int rc = ensure_init_current();
    if (rc) return rc;
    if (nRows && (!d_tree || (nCols && !d_src))) return set_err(B200_EINVAL, "null buffer");
    CK(merkle::build_tree_arity(arity, d_tree, d_src, rs, cs, nCols, nRows, (cudaStream_t)stream,
                                g_native_family.load()),
       "merkletree");
    return B200_OK;
}

static int commit_device_fam(uint64_t *root_host, uint64_t *d_lde, uint64_t *d_tree, const uint64_t *d_trace,
                             int trace_rowmajor, uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t arity,
                             uint64_t *d_scratch, void *stream, int family)
{
    int rc = check_shape(nBits, nBitsExt, nCols, arity);
    if (rc) return rc;
    if ((rc = ensure_init_current())) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t NExt = 1ull << nBitsExt;
    if (!d_tree || (nCols && (!d_lde || !d_trace || !d_scratch))) return set_err(B200_EINVAL, "null buffer");
    CK(ntt::lde(d_lde, d_trace, trace_rowmajor != 0, (uint32_t)nBits, (uint32_t)nBitsExt, nCols, d_scratch, s),
       "lde");
    CK(merkle::build_tree_arity(arity, d_tree, d_lde, 1, NExt, nCols, NExt, s, family), "merkletree");
    if (root_host) {
        const uint64_t total = merkle::tree_num_elements(NExt, arity);
        CK(cudaMemcpyAsync(root_host, d_tree + total - 4, 32, cudaMemcpyDeviceToHost, s), "root D2H");
        CK(cudaStreamSynchronize(s), "sync");
    }
    return B200_OK;
}

extern "C" int b200_commit_device(uint64_t *root_host, uint64_t *d_lde, uint64_t *d_tree, const uint64_t *d_trace,
                                  int trace_rowmajor, uint64_t nBits, uint64_t nBitsExt, uint64_t nCols,
                                  uint64_t arity, uint64_t *d_scratch, void *stream)
{
    return commit_device_fam(root_host, d_lde, d_tree, d_trace, trace_rowmajor, nBits, nBitsExt, nCols, arity,
                             d_scratch, stream, g_native_family.load());
}

extern "C" int b200_permute_device(uint64_t *d_out, const uint64_t *d_in, uint64_t n, uint64_t width, void *stream)
{
    int rc = ensure_init_current();
    if (rc) return rc;
    if (n == 0) return B200_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned tpb = 128, blocks = (unsigned)((n + tpb - 1) / tpb);
    const bool p1 = g_native_family.load() == 1;
    switch (width) {
    case 8:
        if (p1) merkle::permute_kernel<8, 1><<<blocks, tpb, 0, s>>>(d_out, d_in, n);
        else merkle::permute_kernel<8><<<blocks, tpb, 0, s>>>(d_out, d_in, n);
        break;
    case 12:
        if (p1) merkle::permute_kernel<12, 1><<<blocks, tpb, 0, s>>>(d_out, d_in, n);
        else merkle::permute_kernel<12><<<blocks, tpb, 0, s>>>(d_out, d_in, n);
        break;
    case 16:
        if (p1) merkle::permute_kernel<16, 1><<<blocks, tpb, 0, s>>>(d_out, d_in, n);
        else merkle::permute_kernel<16><<<blocks, tpb, 0, s>>>(d_out, d_in, n);
        break;
    default: return set_err(B200_EINVAL, "width must be 8, 12 or 16");
    }
    CK(cudaGetLastError(), "permute");
    return B200_OK;
}

__global__ void lde_rows_kernel(uint64_t *__restrict__ out, const uint64_t *__restrict__ lde, uint64_t NExt,
                                uint64_t ncols, const uint64_t *__restrict__ rows, uint64_t nreq)
{
    const uint64_t i = blockIdx.x, row = rows[i];
    for (uint64_t c = threadIdx.x; c < ncols; c += blockDim.x)
        out[i * ncols + c] = row < NExt ? lde[c * NExt + row] : 0ull;
}

extern "C" int b200_lde_rows_device(uint64_t *d_out, const uint64_t *d_lde, uint64_t NExt, uint64_t nCols,
                                    const uint64_t *d_rows, uint64_t nreq, void *stream)
{
    if (nreq == 0 || nCols == 0) return B200_OK;
    if (nreq > 0x7fffffffULL) return set_err(B200_EINVAL, "too many rows");
    lde_rows_kernel<<<(unsigned)nreq, 128, 0, (cudaStream_t)stream>>>(d_out, d_lde, NExt, nCols, d_rows, nreq);
    CK(cudaGetLastError(), "lde_rows");
    return B200_OK;
}

extern "C" int b200_fill_random_device(uint64_t *d_buf, uint64_t n, uint64_t seed, void *stream)
{
    if (n == 0) return B200_OK;
    const unsigned tpb = 256;
    uint64_t blocks = (n + tpb - 1) / tpb;
    if (blocks > 0x7fffffffULL) return set_err(B200_EINVAL, "buffer too large");
    synth::fill_kernel<<<(unsigned)blocks, tpb, 0, (cudaStream_t)stream>>>(d_buf, n, seed);
    CK(cudaGetLastError(), "fill_random");
    return B200_OK;
}

extern "C" void b200_fill_random_host(uint64_t *buf, uint64_t n, uint64_t seed)
{
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (n < (1u << 16)) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; t++) {
        th.emplace_back([=]() {
            const uint64_t a = n * t / nt, b = n * (t + 1) / nt;
            for (uint64_t i = a; i < b; i++) buf[i] = synth::value(seed, i);
        });
    }
    for (auto &x : th) x.join();
}

extern "C" const char *b200_kernel_names(void)
{
    return "pass16_kernel\ntranspose_kernel\ntranspose_tma_kernel\nleaf_hash_kernel\nnode_kernel\npermute_kernel\nlde_rows_kernel\n"
           "fill_kernel\nimad_probe_kernel\ntranspose_grouped\npass_grouped\nleaf_persistent\n"
           "node_grouped\ngather_roots\npass_fixed_kernel\nopenings_kernel\nbitfield_unpack_kernel\n"
           "unpack_range_kernel\nabsorb_kernel\npass_fixed_grouped\nnode_coop_kernel\ntree_tail_kernel\n"
           "leaf_coop_kernel\n";
}

// ------------------------------------------------------------ host-buffer API ----
struct DevBuf {
    uint64_t *p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(uint64_t words) { return cudaMalloc((void **)&p, (words ? words : 1) * 8); }
};

extern "C" int b200_commit_host(uint64_t *root, uint64_t *lde_out, uint64_t *tree_out, const uint64_t *trace,
                                uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t arity)
{
    int rc = check_shape(nBits, nBitsExt, nCols, arity);
    if (rc) return rc;
    if ((rc = ensure_init_current())) return rc;
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    const uint64_t tsz = merkle::tree_num_elements(NExt, arity);
    DevBuf dt, ds, dl, dtree;
    if (dt.alloc(N * nCols) || ds.alloc(N * nCols) || dl.alloc(NExt * nCols) || dtree.alloc(tsz))
        return set_err(B200_ENOMEM, "device allocation failed");
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    struct SG {
        cudaStream_t s;
        ~SG() { cudaStreamDestroy(s); }
    } sg{s};
    if (N * nCols) CK(cudaMemcpyAsync(dt.p, trace, N * nCols * 8, cudaMemcpyHostToDevice, s), "trace H2D");
    uint64_t r[4];
    rc = b200_commit_device(r, dl.p, dtree.p, dt.p, 1, nBits, nBitsExt, nCols, arity, ds.p, s);
    if (rc) return rc;
    if (root) memcpy(root, r, 32);
    if (lde_out && NExt * nCols) CK(cudaMemcpyAsync(lde_out, dl.p, NExt * nCols * 8, cudaMemcpyDeviceToHost, s), "lde D2H");
    if (tree_out) CK(cudaMemcpyAsync(tree_out, dtree.p, tsz * 8, cudaMemcpyDeviceToHost, s), "tree D2H");
    CK(cudaStreamSynchronize(s), "sync");
    return B200_OK;
}

// ======================================================= reference C ABI ====

static std::atomic<int> g_hash_family{0};  // 0 unset, 1 Poseidon1, 2 Poseidon2

extern "C" void set_hash_family(uint8_t fam)
{
    int expect = 0;
    if (!g_hash_family.compare_exchange_strong(expect, (int)fam) && expect != (int)fam)
        set_err(B200_EFAMILY, "set_hash_family: the hash family cannot change at runtime");
}

static int check_family()
{
    int f = g_hash_family.load();
    if (f == 1 || f == 2) return B200_OK;
    if (f == 0) return set_err(B200_EFAMILY, "hash family not set: call set_hash_family(1 or 2) first");
    return set_err(B200_EFAMILY, "unknown hash family (1 = Poseidon1, 2 = Poseidon2)");
}

extern "C" void init_gpu_setup(uint64_t arity)
{
    (void)arity;
    ensure_init_current();
}

extern "C" bool set_gpu_mode(bool use_gpu)
{
    (void)use_gpu;
    return true;
}

// ------------------------------------------------------------- StarkInfo ----
// stark_info_new (starks_api.hpp:37): the setup's starkinfo JSON, parsed for what the commit path
// and the prover-buffer map need (stark_info.cuh).  The flags keep the reference's meaning; they
// shape the buffer map (gpu, preallocate, recursive, single_use, verify, verify_constraints).
extern "C" void *stark_info_new(char *filename, bool recursive_final, bool recursive, bool verify_constraints,
                                bool verify, bool gpu, bool preallocate, bool single_use)
{
    (void)recursive_final;
    std::string err;
    sinfo::StarkInfo *si = sinfo::from_file(filename, err);
    if (!si) {
        set_err(B200_EINVAL, "stark_info_new: " + err);
        return nullptr;
    }
    si->recursive = recursive;
    si->verify_constraints = verify_constraints;
    si->verify = verify;
    si->gpu = gpu;
    si->preallocate = preallocate;
    si->singleUse = single_use;
    sinfo::buffer_map(*si);
    return si;
}

extern "C" void stark_info_free(void *pStarkInfo)
{
    if (sinfo::StarkInfo *si = sinfo::checked(pStarkInfo)) {
        si->magic = 0;
        delete si;
    }
}

extern "C" uint64_t get_map_total_n(void *pStarkInfo)
{
    const sinfo::StarkInfo *si = sinfo::checked(pStarkInfo);
    return si ? si->mapTotalN : 0;
}

extern "C" uint64_t get_map_total_n_contributions(void *pStarkInfo)
{
    const sinfo::StarkInfo *si = sinfo::checked(pStarkInfo);
    return si ? si->mapTotalNContributions : 0;
}

extern "C" uint64_t get_map_total_n_custom_commits_fixed(void *pStarkInfo)
{
    const sinfo::StarkInfo *si = sinfo::checked(pStarkInfo);
    return si ? si->mapTotalNCustomCommitsFixed : 0;
}

extern "C" uint64_t get_const_size(void *pStarkInfo)
{
    const sinfo::StarkInfo *si = sinfo::checked(pStarkInfo);
    return si ? (1ull << si->nBits) * si->nConstants : 0;
}

extern "C" uint64_t b200_stark_info_offset(void *pStarkInfo, const char *section, int extended)
{
    const sinfo::StarkInfo *si = sinfo::checked(pStarkInfo);
    if (!si || !section) return UINT64_MAX;
    return si->offset(section, extended != 0);
}

extern "C" uint64_t b200_stark_info_value(void *pStarkInfo, const char *name)
{
    const sinfo::StarkInfo *si = sinfo::checked(pStarkInfo);
    if (!si || !name) return UINT64_MAX;
    const std::string n(name);
    if (n == "nBits") return si->nBits;
    if (n == "nBitsExt") return si->nBitsExt;
    if (n == "merkleTreeArity") return si->merkleTreeArity;
    if (n == "lastLevelVerification") return si->lastLevelVerification;
    if (n == "nConstants") return si->nConstants;
    if (n == "nQueries") return si->nQueries;
    if (n == "qDeg") return si->qDeg;
    if (n == "qDim") return si->qDim;
    if (n.rfind("mapSectionsN.", 0) == 0) return si->sectionN(n.substr(13));
    return UINT64_MAX;
}

extern "C" void *b200_stark_shape_new(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t arity)
{
    return sinfo::from_shape(nBits, nBitsExt, nCols, arity);
}

extern "C" void b200_stark_shape_free(void *shape) { stark_info_free(shape); }

// One stream slot: its own device buffers, kept resident after the commit.  `d_aux` is the
// stream's prover buffer laid out by the StarkInfo's map (the reference's d_aux_trace): after a
// commit it holds the column-major trace at ("cm1", false), the LDE at ("cm1", true) and the tree
// at ("mt1", true).  `d_scratch` is the LDE's work area (one column-major copy of the trace).
struct Slot {
    cudaStream_t stream = nullptr;
    cudaStream_t copy = nullptr;  // host-to-device copies of the trace, block by block
    cudaEvent_t h2d_done = nullptr, end = nullptr;
    std::vector<cudaEvent_t> blocks;  // one per column block: that block's copy has landed
    uint64_t *d_aux = nullptr, *d_scratch = nullptr;
    uint64_t cap_aux = 0, cap_scratch = 0;
    uint64_t *d_cm1 = nullptr, *d_lde = nullptr, *d_tree = nullptr;  // views into d_aux (last commit)
    uint64_t aux_words = 0;                                           // extent of d_aux the last commit used
    uint64_t *h_root = nullptr;                                       // pinned 4 words
    uint64_t *user_root = nullptr;
    bool busy = false;
    uint64_t seq = 0;
};

// Word offsets of a commit's regions in the slot's prover buffer.
struct CommitLayout {
    uint64_t cm1_ext, mt1, cm1, words;
};

static CommitLayout commit_layout(uint64_t cm1_ext, uint64_t mt1, uint64_t cm1, uint64_t nBits, uint64_t nBitsExt,
                                  uint64_t nCols, uint64_t arity)
{
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    const uint64_t tsz = merkle::tree_num_elements(NExt, arity);
    CommitLayout l{cm1_ext, mt1, cm1, 0};
    l.words = std::max(cm1_ext + NExt * nCols, std::max(mt1 + tsz, cm1 + N * nCols));
    return l;
}

// the contribution buffer of a commit without a StarkInfo: [cm1 extended][tree][cm1]
static CommitLayout packed_layout(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t arity)
{
    const uint64_t NExt = 1ull << nBitsExt;
    return commit_layout(0, NExt * nCols, NExt * nCols + merkle::tree_num_elements(NExt, arity), nBits, nBitsExt,
                         nCols, arity);
}

struct CommitBuffers {
    int device = 0;
    uint32_t arity = 4;
    std::mutex mu;
    std::vector<Slot> slots;
    uint64_t seq = 0;
    std::atomic<int> error{0};
    // end event of the most recently issued commit: the next commit's kernels wait for it, so
    // commits run one after another on the GPU while the next trace's H2D overlaps them (two
    // commits interleaving would finish together and leave the GPU idle during both next copies)
    cudaEvent_t last_end = nullptr;
    // streaming slot commits (configure_stream_commit_slots): one device block of n slots
    uint64_t *sc_base = nullptr;
    uint64_t sc_slot_bytes = 0;
    std::vector<cudaStream_t> sc_streams;
    std::atomic<int> sc_quiesced{0}, sc_inflight{0};
    // indexed witnesses per (airgroupId, airId): the row layout (b200_register_indexed_air, which
    // stands in for the setup's PackedInfo) and the instruction table (register_instruction_table)
    struct IndexedAir {
        std::vector<uint8_t> col_source;
        uint64_t index_bits = 0;
        uint64_t *d_table = nullptr;
        uint64_t num_entries = 0, words_per_entry = 0;
    };
    std::map<std::pair<uint64_t, uint64_t>, IndexedAir> indexed;
};

// the buffers whose streaming slots stream_commit_pause quiesces (the last configured)
static std::atomic<CommitBuffers *> g_stream_buffers{nullptr};

static int grow(uint64_t *&p, uint64_t &cap, uint64_t words)
{
    if (words <= cap && p) return B200_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc((void **)&p, (words ? words : 1) * 8) != cudaSuccess) return set_err(B200_ENOMEM, "cudaMalloc");
    cap = words;
    return B200_OK;
}

static int slot_create(Slot &s)
{
    CK(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "stream");
    CK(cudaStreamCreateWithFlags(&s.copy, cudaStreamNonBlocking), "stream");
    CK(cudaEventCreateWithFlags(&s.h2d_done, cudaEventDisableTiming), "event");
    CK(cudaEventCreateWithFlags(&s.end, cudaEventDisableTiming), "event");
    CK(cudaMallocHost((void **)&s.h_root, 32), "pinned root");
    return B200_OK;
}

static void slot_destroy(Slot &s)
{
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.copy) cudaStreamSynchronize(s.copy);
    for (cudaEvent_t e : s.blocks) cudaEventDestroy(e);
    for (uint64_t *p : {s.d_aux, s.d_scratch})
        if (p) cudaFree(p);
    if (s.h_root) cudaFreeHost(s.h_root);
    if (s.h2d_done) cudaEventDestroy(s.h2d_done);
    if (s.end) cudaEventDestroy(s.end);
    if (s.stream) cudaStreamDestroy(s.stream);
    if (s.copy) cudaStreamDestroy(s.copy);
    s = Slot{};
}

extern "C" void *gen_device_buffers(uint32_t node_rank, uint32_t node_size, const int32_t *numa_nodes,
                                    uint32_t arity, uint32_t max_n_bits_ext)
{
    (void)node_rank;
    (void)node_size;
    (void)numa_nodes;
    (void)max_n_bits_ext;
    if (ensure_init_current()) return nullptr;
    auto *b = new CommitBuffers();
    cudaGetDevice(&b->device);
    b->arity = arity;
    b->slots.resize(2);
    for (auto &s : b->slots)
        if (slot_create(s)) {
            for (auto &x : b->slots) slot_destroy(x);
            delete b;
            return nullptr;
        }
    return b;
}

extern "C" void free_device_buffers(void *d_buffers)
{
    auto *b = (CommitBuffers *)d_buffers;
    if (!b) return;
    for (auto &s : b->slots) slot_destroy(s);
    for (cudaStream_t t : b->sc_streams) {
        cudaStreamSynchronize(t);
        cudaStreamDestroy(t);
    }
    if (b->sc_base) cudaFree(b->sc_base);
    for (auto &kv : b->indexed)
        if (kv.second.d_table) cudaFree(kv.second.d_table);
    CommitBuffers *expect = b;
    g_stream_buffers.compare_exchange_strong(expect, nullptr);
    delete b;
}

// A commit that failed on the device is reported on the buffers object (and its root left zero).
static void harvest(CommitBuffers *b, Slot &s)
{
    if (!s.busy) return;
    const cudaError_t e = cudaEventSynchronize(s.end);
    if (e == cudaSuccess) {
        if (s.user_root) memcpy(s.user_root, s.h_root, 32);
    } else {
        b->error = cuda_err(e, "commit on the device");
        if (s.user_root) memset(s.user_root, 0, 32);
    }
    s.busy = false;
}

extern "C" uint64_t gen_device_streams(void *d_buffers, uint64_t n_streams, uint64_t n_recursive_streams,
                                       const uint64_t *auxTraceSizes, uint64_t maxSizeProverBufferAggregation,
                                       uint64_t maxProofSize, uint64_t merkleTreeArity)
{
    (void)n_recursive_streams;
    (void)auxTraceSizes;
    (void)maxSizeProverBufferAggregation;
    (void)maxProofSize;
    auto *b = (CommitBuffers *)d_buffers;
    if (!b || n_streams == 0 || n_streams > 64) return 0;
    std::lock_guard<std::mutex> lk(b->mu);
    cudaSetDevice(b->device);
    if (merkleTreeArity) b->arity = (uint32_t)merkleTreeArity;
    for (auto &s : b->slots) harvest(b, s);
    b->last_end = nullptr;  // every slot is idle; slots may be destroyed below
    while (b->slots.size() > n_streams) {
        slot_destroy(b->slots.back());
        b->slots.pop_back();
    }
    while (b->slots.size() < n_streams) {
        b->slots.emplace_back();
        if (slot_create(b->slots.back())) {
            b->slots.pop_back();
            break;
        }
    }
    return b->slots.size();
}

// Column blocks of the pipelined commit, as start columns (starts.back() == nCols): when the
// trace is large enough for the overlap to matter, a 16-column first block (nothing hides its
// copy: the kernels start once it has landed; 128-byte row segments still copy at 47 GB/s), then
// blocks of 24 and 48 columns, then 64-column blocks (512-byte row segments, which a 2-D copy
// moves at the full 55 GB/s).  On an idle device the kernels of the blocks already landed (LDE
// plus the chunked sponge, ~1.1 ms per 2^22-row column against ~0.6 ms of copy) must outlast the
// next block's copy, or the GPU waits: after 16 columns that allows about 28 more, after 40
// about 49 more.
static void commit_blocks(uint64_t nBits, uint64_t nCols, std::vector<uint64_t> &starts)
{
    starts.assign(1, 0);
    if (nBits >= 16 && nCols >= 128) {
        starts.push_back(16);
        starts.push_back(40);
        for (uint64_t c = 88; c < nCols; c += 64) starts.push_back(c);
    }
    if (nCols) starts.push_back(nCols);
}

// Device buffers of one pipelined commit (pipelined_commit).  `staging` (N * nCols words) receives
// the row-major column blocks, block [c0, c0 + cb) at staging + c0 * N with row pitch cb; `cm1`
// (N * nCols) receives the column-major trace and `scratch` (N * nCols) is the LDE's work area,
// which may be cm1 itself (the LDE then runs in place on the transposed trace).
struct PipeBuffers {
    uint64_t *staging = nullptr, *cm1 = nullptr, *scratch = nullptr, *lde = nullptr, *tree = nullptr;
    uint64_t *h_root = nullptr;  // pinned 4 words for the root (null: left in the tree)
};

// H2D + LDE + tree (+ root D2H) of a row-major host trace, pipelined over column blocks: the blocks
// cross PCIe on `copy`, each a 2-D copy into its staging block; `comp` transposes each block into
// cm1 as soon as it has landed and extends it into the LDE, so the LDE of a block overlaps the copy
// of the next, then hashes the rows once every column is extended.  `copy` first waits for
// `copy_after` and `comp` for `comp_after` (either may be null).  block_ev needs one event per
// column block (commit_blocks); h2d_done (nullable) is recorded after the last copy and
// comp_started (nullable) on `comp` once the first block has landed and comp_after has passed.
//
// With `idle` (nothing else runs on the device, so the copy is exposed), an arity-4 commit hashes
// its rows while the later column blocks are still crossing: the row sponge in 12-column chunks
// (stream::absorb_kernel, the 4-word state carried in tree level 0), each chunk as soon as its
// columns are extended.  Same sponge, same digests.
static int pipelined_commit(const uint64_t *trace, uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t arity,
                            int fam, const PipeBuffers &pb, cudaStream_t copy, cudaStream_t comp,
                            std::vector<cudaEvent_t> &block_ev, cudaEvent_t h2d_done, cudaEvent_t copy_after,
                            cudaEvent_t comp_after, bool idle, cudaEvent_t comp_started = nullptr)
{
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    const uint64_t tsz = merkle::tree_num_elements(NExt, arity);
    std::vector<uint64_t> starts;
    commit_blocks(nBits, nCols, starts);
    const uint64_t nblk = starts.size() - 1;
    while (block_ev.size() < nblk) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        block_ev.push_back(e);
    }
    if (copy_after) CK(cudaStreamWaitEvent(copy, copy_after, 0), "copy order");
    for (uint64_t k = 0; k < nblk; k++) {
        const uint64_t c0 = starts[k], cb = starts[k + 1] - c0;
        if (cb == nCols)
            CK(cudaMemcpyAsync(pb.staging, trace, N * nCols * 8, cudaMemcpyHostToDevice, copy), "trace H2D");
        else
            CK(cudaMemcpy2DAsync(pb.staging + c0 * N, cb * 8, trace + c0, nCols * 8, cb * 8, N, cudaMemcpyHostToDevice,
                                 copy),
               "trace block H2D");
        CK(cudaEventRecord(block_ev[k], copy), "event");
    }
    if (h2d_done) CK(cudaEventRecord(h2d_done, copy), "event");
    const bool chunked = idle && arity == 4 && nblk > 1;
    uint64_t next_chunk = 0;
    if (comp_after) CK(cudaStreamWaitEvent(comp, comp_after, 0), "order commits");
    for (uint64_t k = 0; k < nblk; k++) {
        const uint64_t c0 = starts[k], cb = starts[k + 1] - c0;
        CK(cudaStreamWaitEvent(comp, block_ev[k], 0), "block landed");
        if (k == 0 && comp_started) CK(cudaEventRecord(comp_started, comp), "event");
        {
            prof::Scope ps(prof::TRANSPOSE, comp);
            CK(ntt::transpose(pb.cm1 + c0 * N, pb.staging + c0 * N, N, cb, N, comp), "transpose");
        }
        CK(ntt::lde(pb.lde + c0 * NExt, pb.cm1 + c0 * N, false, (uint32_t)nBits, (uint32_t)nBitsExt, cb,
                    pb.scratch + c0 * N, comp),
           "lde");
        if (chunked) {
            const uint64_t avail = k + 1 == nblk ? nCols : c0 + cb;  // columns extended so far
            prof::Scope ps(prof::LEAF_HASH, comp);
            for (; next_chunk * stream::RATE < nCols; next_chunk++) {
                const uint64_t a0 = next_chunk * stream::RATE;
                const uint32_t cc = (uint32_t)std::min<uint64_t>(stream::RATE, nCols - a0);
                if (a0 + cc > avail) break;
                const unsigned grid = (unsigned)((NExt + merkle::TPB - 1) / merkle::TPB);
                if (fam == 1)
                    stream::absorb_kernel<1><<<grid, merkle::TPB, 0, comp>>>(pb.tree, pb.lde + a0 * NExt, cc,
                                                                             next_chunk == 0, NExt);
                else
                    stream::absorb_kernel<2><<<grid, merkle::TPB, 0, comp>>>(pb.tree, pb.lde + a0 * NExt, cc,
                                                                             next_chunk == 0, NExt);
                prof::count();
                CK(cudaGetLastError(), "absorb");
            }
        }
    }
    if (chunked) {
        const cudaError_t e = fam == 1 ? merkle::build_levels<16, 1>(pb.tree, NExt, comp)
                                       : merkle::build_levels<16, 2>(pb.tree, NExt, comp);
        CK(e, "tree levels");
    } else
        CK(merkle::build_tree_arity(arity, pb.tree, pb.lde, 1, NExt, nCols, NExt, comp, fam), "merkletree");
    if (pb.h_root)
        CK(cudaMemcpyAsync(pb.h_root, pb.tree + tsz - 4, 32, cudaMemcpyDeviceToHost, comp), "root D2H");
    return B200_OK;
}

// Enqueue H2D + LDE + tree + root D2H for a row-major host trace on a slot, into the regions of the
// slot's prover buffer that `lay` names (pipelined_commit over the slot's copy and compute streams).
//
// The staging area is the top N * nCols words of the ("cm1", true) region, as the reference stages
// its trace in that region (commit_witness_gpu, starks_api.cu:1651-1659).  The LDE of the blocks up
// to column x writes words [0, x * NExt) of the region, below every later block's staging, which
// starts at (NExt - N) * nCols + x * N >= x * NExt for x <= nCols; so copies running ahead never
// land on extended columns, and a block's own staging is overwritten only after its transpose.
// The transposed trace stays in ("cm1", false) (the LDE reads it into the scratch), as the
// reference's preserve_src LDE leaves it.
//
// The compute stream also waits for the previously issued commit to end (see
// CommitBuffers::last_end); the copy stream only for this slot's previous commit (which may still
// read the staging area).  With an earlier commit still running, this commit's copy hides under it
// and its kernels wait for it anyway; with the device idle the copy is exposed and the rows are
// hashed in chunks while the later blocks cross.
static int slot_commit(CommitBuffers *b, Slot &s, const uint64_t *trace, uint64_t nBits, uint64_t nBitsExt,
                       uint64_t nCols, uint64_t arity, const CommitLayout &lay)
{
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    int rc;
    if ((rc = grow(s.d_aux, s.cap_aux, lay.words)) || (rc = grow(s.d_scratch, s.cap_scratch, N * nCols))) return rc;
    s.d_lde = s.d_aux + lay.cm1_ext;
    s.d_tree = s.d_aux + lay.mt1;
    s.d_cm1 = s.d_aux + lay.cm1;
    s.aux_words = lay.words;
    PipeBuffers pb;
    pb.staging = s.d_lde + (NExt - N) * nCols;
    pb.cm1 = s.d_cm1;
    pb.scratch = s.d_scratch;
    pb.lde = s.d_lde;
    pb.tree = s.d_tree;
    pb.h_root = s.h_root;
    const bool idle = !b->last_end || cudaEventQuery(b->last_end) == cudaSuccess;
    cudaEvent_t after = b->last_end && b->last_end != s.end ? b->last_end : nullptr;
    if ((rc = pipelined_commit(trace, nBits, nBitsExt, nCols, arity, g_hash_family.load(), pb, s.copy, s.stream,
                               s.blocks, s.h2d_done, s.end, after, idle)))
        return rc;
    CK(cudaEventRecord(s.end, s.stream), "event");
    b->last_end = s.end;
    return B200_OK;
}

// pSetupCtx is proofman's SetupC {p_stark_info, p_expressions_bin} (common/src/setup.rs:45-57), whose
// p_stark_info came from stark_info_new or b200_stark_shape_new.
extern "C" uint64_t commit_witness(void *pSetupCtx, void *params, uint64_t instanceId, uint64_t airgroupId,
                                   uint64_t airId, void *root, void *d_buffers, char *customCommitsFixedPath)
{
    (void)instanceId;
    (void)airgroupId;
    (void)airId;
    (void)customCommitsFixedPath;
    auto *b = (CommitBuffers *)d_buffers;
    auto *setup = (const B200SetupC *)pSetupCtx;
    auto *sp = (const B200StepsParams *)params;
    if (!b || !setup || !sp) {
        set_err(B200_EINVAL, "commit_witness: null argument");
        if (b) b->error = B200_EINVAL;
        return UINT64_MAX;
    }
    const sinfo::StarkInfo *si = sinfo::checked(setup->p_stark_info);
    if (!si) {
        b->error = set_err(B200_EINVAL, "commit_witness: pSetupCtx->p_stark_info is not a StarkInfo of this library "
                                        "(stark_info_new / b200_stark_shape_new)");
        return UINT64_MAX;
    }
    if (si->verificationHashType != "GL") {
        b->error = set_err(B200_EINVAL, "commit_witness: only the Goldilocks (GL) Merkle commit is provided");
        return UINT64_MAX;
    }
    const uint64_t nCols = si->sectionN("cm1"), arity = si->merkleTreeArity;
    int rc = check_family();
    if (!rc) rc = check_shape(si->nBits, si->nBitsExt, nCols, arity);
    if (!rc && (si->offset("cm1", true) == UINT64_MAX || si->offset("mt1", true) == UINT64_MAX ||
                si->offset("cm1", false) == UINT64_MAX))
        rc = set_err(B200_EINVAL, "commit_witness: the StarkInfo has no stage-1 buffer map (verifier layout?)");
    if (rc) {
        b->error = rc;
        return UINT64_MAX;
    }
    const CommitLayout lay = commit_layout(si->offset("cm1", true), si->offset("mt1", true), si->offset("cm1", false),
                                           si->nBits, si->nBitsExt, nCols, arity);
    std::lock_guard<std::mutex> lk(b->mu);
    cudaSetDevice(b->device);
    // a free slot, else the oldest in flight (harvested first)
    size_t pick = b->slots.size();
    for (size_t i = 0; i < b->slots.size(); i++)
        if (!b->slots[i].busy) {
            pick = i;
            break;
        }
    if (pick == b->slots.size()) {
        pick = 0;
        for (size_t i = 1; i < b->slots.size(); i++)
            if (b->slots[i].seq < b->slots[pick].seq) pick = i;
        harvest(b, b->slots[pick]);
    }
    Slot &s = b->slots[pick];
    rc = slot_commit(b, s, sp->trace, si->nBits, si->nBitsExt, nCols, arity, lay);
    if (rc) {
        b->error = rc;
        return UINT64_MAX;
    }
    s.user_root = (uint64_t *)root;
    s.busy = true;
    s.seq = ++b->seq;
    return pick;
}

// The prover buffer of a stream slot (the reference's d_aux_trace of that stream) and the words its
// last commit used: the trace, LDE and tree sit at the StarkInfo's mapOffsets.  Valid once the
// slot's commit has been harvested.
extern "C" int b200_commit_buffers_aux(void *d_buffers, uint64_t stream_id, uint64_t **d_aux, uint64_t *words)
{
    auto *b = (CommitBuffers *)d_buffers;
    if (!b) return set_err(B200_EINVAL, "null buffers");
    std::lock_guard<std::mutex> lk(b->mu);
    if (stream_id >= b->slots.size()) return set_err(B200_EINVAL, "stream id out of range");
    if (d_aux) *d_aux = b->slots[stream_id].d_aux;
    if (words) *words = b->slots[stream_id].aux_words;
    return B200_OK;
}

extern "C" void get_stream_proofs(void *d_buffers)
{
    auto *b = (CommitBuffers *)d_buffers;
    if (!b) return;
    std::lock_guard<std::mutex> lk(b->mu);
    for (auto &s : b->slots) harvest(b, s);
}

extern "C" void get_stream_proofs_non_blocking(void *d_buffers)
{
    auto *b = (CommitBuffers *)d_buffers;
    if (!b) return;
    std::lock_guard<std::mutex> lk(b->mu);
    for (auto &s : b->slots)
        if (s.busy && cudaEventQuery(s.end) != cudaErrorNotReady) harvest(b, s);
}

extern "C" uint32_t register_host_memory(void *ptr, uint64_t size)
{
    if (!ptr || size == 0) return 0;
    if (cudaHostRegister(ptr, size, cudaHostRegisterPortable) != cudaSuccess) {
        cudaGetLastError();  // a refused registration leaves no sticky error
        return 0;
    }
    return 1;
}

extern "C" void unregister_host_memory(void *ptr)
{
    if (ptr && cudaHostUnregister(ptr) != cudaSuccess) cudaGetLastError();
}

extern "C" void wait_trace_h2d_done(void *d_buffers, uint64_t stream_id)
{
    auto *b = (CommitBuffers *)d_buffers;
    if (!b) return;
    Slot *s = nullptr;
    {
        std::lock_guard<std::mutex> lk(b->mu);
        if (stream_id < b->slots.size()) s = &b->slots[stream_id];
    }
    if (s && s->h2d_done) cudaEventSynchronize(s->h2d_done);
}

extern "C" int b200_buffers_error(void *d_buffers)
{
    auto *b = (CommitBuffers *)d_buffers;
    return b ? b->error.load() : B200_EINVAL;
}

static bool write_words(std::ofstream &f, const uint64_t *p, uint64_t n)
{
    f.write((const char *)p, (std::streamsize)(n * 8));
    return (bool)f;
}

extern "C" void write_custom_commit(void *root, uint64_t arity, uint64_t nBits, uint64_t nBitsExt, uint64_t nCols,
                                   void *d_buffers, void *buffer, char *bufferFile)
{
    auto *b = (CommitBuffers *)d_buffers;
    uint64_t *r = (uint64_t *)root;
    if (r) memset(r, 0, 32);
    int rc = check_family();
    if (!rc) rc = check_shape(nBits, nBitsExt, nCols, arity);
    if (!rc && (!root || !buffer)) rc = set_err(B200_EINVAL, "write_custom_commit: null argument");
    bool own = false;
    if (!rc && !b) {
        b = (CommitBuffers *)gen_device_buffers(0, 1, nullptr, (uint32_t)arity, (uint32_t)nBitsExt);
        own = true;
        if (!b) rc = B200_ENOMEM;
    }
    if (rc) {
        if (b) b->error = rc;
        return;
    }
    {
        std::lock_guard<std::mutex> lk(b->mu);
        cudaSetDevice(b->device);
        Slot &s = b->slots[0];
        harvest(b, s);
        const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
        const uint64_t tsz = merkle::tree_num_elements(NExt, arity);
        rc = slot_commit(b, s, (const uint64_t *)buffer, nBits, nBitsExt, nCols, arity,
                         packed_layout(nBits, nBitsExt, nCols, arity));
        if (!rc && cudaStreamSynchronize(s.stream) != cudaSuccess) rc = set_err(B200_ECUDA, "commit failed");
        if (!rc) memcpy(r, s.h_root, 32);
        if (!rc && bufferFile && bufferFile[0]) {
            std::vector<uint64_t> host((N + NExt) * nCols + tsz);
            // source column-major (the transposed trace the commit left in its ("cm1", false) region,
            // canonicalised here), then LDE and nodes
            cudaMemcpy(host.data(), s.d_cm1, N * nCols * 8, cudaMemcpyDeviceToHost);
            for (uint64_t i = 0; i < N * nCols; i++)
                if (host[i] >= GL_P) host[i] -= GL_P;
            cudaMemcpy(host.data() + N * nCols, s.d_lde, NExt * nCols * 8, cudaMemcpyDeviceToHost);
            cudaMemcpy(host.data() + (N + NExt) * nCols, s.d_tree, tsz * 8, cudaMemcpyDeviceToHost);
            std::ofstream f(bufferFile, std::ios::binary | std::ios::trunc);
            if (!f || !write_words(f, r, 4) || !write_words(f, host.data(), host.size()))
                rc = set_err(B200_EINVAL, std::string("cannot write ") + bufferFile);
        }
    }
    if (rc) b->error = rc;
    if (own) free_device_buffers(b);
}

extern "C" uint64_t get_const_tree_size(void *pStarkInfo)
{
    const sinfo::StarkInfo *si = sinfo::checked(pStarkInfo);
    if (!si || si->merkleTreeArity < 2 || si->verificationHashType != "GL") return 0;
    const uint64_t NExt = 1ull << si->nBitsExt;
    return NExt * si->nConstants + si->numNodesMT(NExt);
}

// pStarkInfo: from stark_info_new (nConstants columns) or b200_stark_shape_new (nCols columns).
extern "C" void calculate_const_tree(void *pStarkInfo, void *pConstPolsAddress, void *pConstTree,
                                     void *unified_buffer_gpu)
{
    const sinfo::StarkInfo *si = sinfo::checked(pStarkInfo);
    if (!si || !pConstPolsAddress || !pConstTree) {
        set_err(B200_EINVAL, "calculate_const_tree: null argument or not a StarkInfo of this library");
        return;
    }
    struct {
        uint64_t nBits, nBitsExt, nCols, arity;
    } const shape{si->nBits, si->nBitsExt, si->nConstants, si->merkleTreeArity}, *sh = &shape;
    if (check_family() || check_shape(sh->nBits, sh->nBitsExt, sh->nCols, sh->arity)) return;
    if (ensure_init_current()) return;
    const uint64_t N = 1ull << sh->nBits, NExt = 1ull << sh->nBitsExt, nCols = sh->nCols;
    const uint64_t tsz = merkle::tree_num_elements(NExt, sh->arity);
    const uint64_t total = NExt * nCols + tsz;
    DevBuf tree_own, tr, sc;
    uint64_t *d_tree = (uint64_t *)unified_buffer_gpu;
    if (!d_tree) {
        if (tree_own.alloc(total)) {
            set_err(B200_ENOMEM, "cudaMalloc");
            return;
        }
        d_tree = tree_own.p;
    }
    if (tr.alloc(N * nCols) || sc.alloc(N * nCols)) {
        set_err(B200_ENOMEM, "cudaMalloc");
        return;
    }
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        set_err(B200_ECUDA, "calculate_const_tree: stream creation failed");
        return;
    }
    cudaError_t e = cudaSuccess;
    if (N * nCols) e = cudaMemcpyAsync(tr.p, pConstPolsAddress, N * nCols * 8, cudaMemcpyHostToDevice, s);
    int rc = e == cudaSuccess ? B200_OK : set_err(B200_ECUDA, "calculate_const_tree: trace copy failed");
    if (!rc)
        rc = commit_device_fam(nullptr, d_tree, d_tree + NExt * nCols, tr.p, 1, sh->nBits, sh->nBitsExt, nCols,
                               sh->arity, sc.p, s, g_hash_family.load());
    if (!rc && cudaMemcpyAsync(pConstTree, d_tree, total * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        rc = set_err(B200_ECUDA, "calculate_const_tree: result copy failed");
    // the stream is drained before the device buffers are freed, whatever happened above
    if (cudaStreamSynchronize(s) != cudaSuccess && !rc) set_err(B200_ECUDA, "calculate_const_tree: commit failed");
    cudaStreamDestroy(s);
}

// ------------------------------------------------------------- profiling ----
extern "C" void b200_timing_enable(int on) { prof::g_enabled.store(on ? 1 : 0); }
extern "C" void b200_timing_reset(void) { prof::reset(); }
extern "C" int b200_timing_get(int category, double *total_ms, uint64_t *count)
{
    if (category < 0 || category >= prof::NCAT) return set_err(B200_EINVAL, "bad timing category");
    prof::collect();
    std::lock_guard<std::mutex> lk(prof::g_mu);
    if (total_ms) *total_ms = prof::g_ms[category];
    if (count) *count = prof::g_count[category];
    return B200_OK;
}
extern "C" const char *b200_timing_name(int category)
{
    return (category >= 0 && category < prof::NCAT) ? prof::kCatNames[category] : "";
}
extern "C" uint64_t b200_launch_count(void) { return prof::g_launches.load(); }

extern "C" int b200_set_transpose_tma(int on) { return ntt::transpose_tma_enabled().exchange(on ? 1 : 0); }

// the TMA transposes' error flag on the current device (1: a tile copy did not land within the
// kernel's wait bound), reset to 0
extern "C" int b200_tma_wait_errors(void)
{
    int v = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&v, g_tma_error, sizeof(int)) != cudaSuccess) return cuda_err(cudaGetLastError(), "flag");
    CK(cudaMemcpyToSymbol(g_tma_error, &zero, sizeof(int)), "flag reset");
    return v;
}

__global__ void __launch_bounds__(256) imad_probe_kernel(uint32_t *out, uint64_t iters, uint32_t seed)
{
    uint32_t x[8];
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = seed + threadIdx.x * 8 + j;
    const uint32_t a = 0x9e3779b9u ^ seed, c = 0x7f4a7c15u;
    for (uint64_t i = 0; i < iters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x[j]) : "r"(a), "r"(c));
            asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(x[j + 1]) : "r"(a), "r"(c));
        }
    }
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) acc ^= x[j];
    if (acc == 0x12345678u) out[blockIdx.x] = acc;  // keeps the chains live
}

extern "C" int b200_probe_imad(uint64_t blocks, uint64_t iters, double *gimad_per_s)
{
    int rc = ensure_init_current();
    if (rc) return rc;
    if (blocks == 0 || blocks > 0x7fffffffULL) return set_err(B200_EINVAL, "bad block count");
    DevBuf out;
    if (out.alloc(blocks)) return set_err(B200_ENOMEM, "cudaMalloc");
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0), "event");
    CK(cudaEventCreate(&e1), "event");
    imad_probe_kernel<<<(unsigned)blocks, 256>>>((uint32_t *)out.p, iters / 8 + 1, 1);  // warm-up
    CK(cudaEventRecord(e0), "event");
    imad_probe_kernel<<<(unsigned)blocks, 256>>>((uint32_t *)out.p, iters, 2);
    CK(cudaEventRecord(e1), "event");
    CK(cudaEventSynchronize(e1), "probe");
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (gimad_per_s) *gimad_per_s = (double)blocks * 256.0 * 8.0 * (double)iters / (ms * 1e-3) / 1e9;
    return B200_OK;
}


// ---------------------------------------------------- batched commit and server ----
#include "batch_api.cuh"
#include "server.cuh"

// ------------------------------------------------------------- query openings ----
#include "query.cuh"

extern "C" uint64_t b200_query_proof_words(uint64_t NExt, uint64_t nCols, uint64_t arity,
                                           uint64_t last_level_verification)
{
    if (arity < 2 || arity > 4 || NExt == 0) return 0;
    return query::proof_words(NExt, nCols, arity, last_level_verification);
}

extern "C" int b200_query_openings_device(uint64_t *d_out, const uint64_t *d_lde, uint64_t NExt, uint64_t nCols,
                                          const uint64_t *d_tree, uint64_t arity, uint64_t last_level_verification,
                                          const uint64_t *d_rows, uint64_t nQueries, void *stream)
{
    if (arity < 2 || arity > 4) return set_err(B200_EINVAL, "arity must be 2, 3 or 4");
    if (NExt == 0) return set_err(B200_EINVAL, "empty tree");
    if (nQueries == 0) return B200_OK;
    if (nQueries > 0x7fffffffULL) return set_err(B200_EINVAL, "too many queries");
    if (!d_out || !d_tree || !d_rows || (nCols && !d_lde)) return set_err(B200_EINVAL, "null buffer");
    const uint64_t levels = query::proof_levels(NExt, arity, last_level_verification);
    const uint64_t words = nCols + levels * (arity - 1) * 4;
    query::openings_kernel<<<(unsigned)nQueries, 256, 0, (cudaStream_t)stream>>>(d_out, d_lde, NExt, nCols, d_tree,
                                                                                 arity, levels, d_rows, words);
    CK(cudaGetLastError(), "query openings");
    return B200_OK;
}

// ------------------------------------------------------------ Q-stage commit ----
extern "C" uint64_t b200_q_scratch_words(uint64_t nBitsExt, uint64_t qDim) { return (1ull << nBitsExt) * qDim; }

extern "C" int b200_commit_q_device(uint64_t *root_host, uint64_t *d_cmq, uint64_t *d_tree, const uint64_t *d_q,
                                    int q_rowmajor, uint64_t nBits, uint64_t nBitsExt, uint64_t qDeg, uint64_t qDim,
                                    uint64_t arity, uint64_t *d_scratch, void *stream)
{
    int rc = check_shape(nBits, nBitsExt, qDeg * qDim, arity);
    if (rc) return rc;
    if (qDeg > (1ull << (nBitsExt - nBits))) return set_err(B200_EINVAL, "qDeg above NExt / N");
    if ((rc = ensure_init_current())) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t NExt = 1ull << nBitsExt, ncols = qDeg * qDim;
    if (!d_tree || (ncols && (!d_cmq || !d_q || !d_scratch))) return set_err(B200_EINVAL, "null buffer");
    CK(ntt::lde_q(d_cmq, d_q, q_rowmajor != 0, (uint32_t)nBits, (uint32_t)nBitsExt, (uint32_t)qDeg, (uint32_t)qDim,
                  d_scratch, s),
       "Q extension");
    CK(merkle::build_tree_arity(arity, d_tree, d_cmq, 1, NExt, ncols, NExt, s, g_native_family.load()), "merkletree");
    if (root_host) {
        const uint64_t total = merkle::tree_num_elements(NExt, arity);
        CK(cudaMemcpyAsync(root_host, d_tree + total - 4, 32, cudaMemcpyDeviceToHost, s), "root D2H");
        CK(cudaStreamSynchronize(s), "sync");
    }
    return B200_OK;
}

// ------------------------------------------------------------ plan autotuner ----
// Times lde() under each candidate plan (largest first window kf, largest later window kr,
// both in 8..12) on a probe of min(nCols, 256) columns of seeded data, interleaving each
// candidate's runs with the default plan's, and keeps a candidate only if it beats the default by
// more than 3 % (probe timings of plans that differ by less are noise, and a narrower probe can
// rank plans differently from the full width).  Untimed set-up; every plan computes the same values.
extern "C" int b200_autotune_lde(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, double *best_ms,
                                 uint32_t *kfirst, uint32_t *krest)
{
    int rc = check_shape(nBits, nBitsExt, nCols, 4);
    if (rc) return rc;
    if ((rc = ensure_init_current())) return rc;
    const uint64_t probe = nCols < 256 ? (nCols ? nCols : 1) : 256;
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    uint64_t *d_trace = nullptr, *d_lde = nullptr, *d_scr = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto cleanup = [&]() {
        if (d_trace) cudaFree(d_trace);
        if (d_lde) cudaFree(d_lde);
        if (d_scr) cudaFree(d_scr);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (s) cudaStreamDestroy(s);
    };
    if (cudaMalloc(&d_trace, N * probe * 8) != cudaSuccess || cudaMalloc(&d_lde, NExt * probe * 8) != cudaSuccess ||
        cudaMalloc(&d_scr, N * probe * 8) != cudaSuccess || cudaStreamCreate(&s) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cleanup();
        cudaGetLastError();
        return set_err(B200_ENOMEM, "autotune buffers");
    }
    synth::fill_kernel<<<(unsigned)((N * probe + 255) / 256), 256, 0, s>>>(d_trace, N * probe, 99);
    // best of three runs of plan t (after one warm-up); < 0 on a CUDA error
    auto time_plan = [&](ntt::Tune t) -> double {
        ntt::set_tuned((uint32_t)nBits, (uint32_t)nBitsExt, nCols, t);
        float best_ms_t = 1e30f;
        for (int it = 0; it < 4; it++) {
            cudaEventRecord(e0, s);
            if (ntt::lde(d_lde, d_trace, true, (uint32_t)nBits, (uint32_t)nBitsExt, probe, d_scr, s) != cudaSuccess)
                return -1;
            cudaEventRecord(e1, s);
            float ms = 0;
            if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
                return -1;
            if (it > 0 && ms < best_ms_t) best_ms_t = ms;
        }
        return best_ms_t;
    };
    const ntt::Tune def{};
    ntt::Tune bt = def;
    double best = 1e30, best_ratio = 1.0;
    // the windows a plan produces (candidates with the default's windows need no run)
    auto windows = [&](ntt::Tune t) {
        std::vector<uint32_t> v;
        ntt::Window w[8];
        int n1 = nBits ? ntt::plan_windows(0, (uint32_t)nBits, w, 8, t.kfirst, t.krest) : 0;
        for (int i = 0; i < n1; i++) v.insert(v.end(), {w[i].s0, w[i].k, w[i].lgL});
        v.push_back(99);
        int n2 = ntt::plan_windows((uint32_t)(nBitsExt - nBits), (uint32_t)nBitsExt, w, 8, t.kfirst, t.krest);
        for (int i = 0; i < n2; i++) v.insert(v.end(), {w[i].s0, w[i].k, w[i].lgL});
        if (n1 < 0 || n2 < 0) v.clear();
        return v;
    };
    const std::vector<uint32_t> wdef = windows(def);
    for (uint32_t kf = 8; kf <= NTT_KMAX; kf++) {
        for (uint32_t kr = 8; kr <= NTT_KMAX; kr++) {
            const std::vector<uint32_t> wc = windows(ntt::Tune{kf, kr});
            if (wc.empty() || wc == wdef) continue;
            const double td = time_plan(def), tc = time_plan(ntt::Tune{kf, kr});
            if (td < 0 || tc < 0) {
                ntt::set_tuned((uint32_t)nBits, (uint32_t)nBitsExt, nCols, def);
                cleanup();
                return set_err(B200_ECUDA, "autotune run failed");
            }
            if (td < best && bt.kfirst == def.kfirst && bt.krest == def.krest) best = td;
            const double ratio = tc / td;
            if (ratio < 0.97 && ratio < best_ratio) {
                best_ratio = ratio;
                bt = ntt::Tune{kf, kr};
                best = tc;
            }
        }
    }
    if (best > 1e29) best = time_plan(bt);  // every candidate had the default's windows
    ntt::set_tuned((uint32_t)nBits, (uint32_t)nBitsExt, nCols, bt);
    cleanup();
    if (best_ms) *best_ms = best;
    if (kfirst) *kfirst = bt.kfirst;
    if (krest) *krest = bt.krest;
    return B200_OK;
}

extern "C" void b200_autotune_get(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint32_t *kfirst,
                                  uint32_t *krest)
{
    const ntt::Tune t = ntt::tuned((uint32_t)nBits, (uint32_t)nBitsExt, nCols);
    if (kfirst) *kfirst = t.kfirst;
    if (krest) *krest = t.krest;
}

extern "C" void b200_autotune_set(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint32_t kfirst, uint32_t krest)
{
    ntt::set_tuned((uint32_t)nBits, (uint32_t)nBitsExt, nCols, ntt::Tune{kfirst, krest});
}

// table file: one line per tuned key, "key kfirst krest"
extern "C" int b200_autotune_save(const char *path)
{
    std::lock_guard<std::mutex> lk(ntt::tune_mu());
    std::ofstream f(path);
    if (!f) return set_err(B200_EINVAL, "cannot open plan file for writing");
    for (const auto &kv : ntt::tune_table()) f << kv.first << " " << kv.second.kfirst << " " << kv.second.krest << "\n";
    return f ? B200_OK : set_err(B200_EINVAL, "plan file write failed");
}

extern "C" int b200_autotune_load(const char *path)
{
    std::ifstream f(path);
    if (!f) return set_err(B200_EINVAL, "cannot open plan file");
    uint64_t key;
    uint32_t kf, kr;
    std::lock_guard<std::mutex> lk(ntt::tune_mu());
    while (f >> key >> kf >> kr) {
        if (kf < 1 || kf > NTT_KMAX || kr < 1 || kr > NTT_KMAX) return set_err(B200_EINVAL, "bad plan entry");
        ntt::tune_table()[key] = ntt::Tune{kf, kr};
    }
    return B200_OK;
}

// ------------------------------------------------------ packed-witness commit ----
#include "unpack.cuh"

extern "C" uint64_t b200_packed_words_per_row(const uint32_t *col_bits, uint64_t nCols)
{
    return (unpack::packed_bits(col_bits, nCols) + 63) / 64;
}

// Commit of a bit-packed row-major witness (the reference's packed trace: PackedInfo and the
// unpack kernel, starks_gpu.cu:49-103; commit_witness_gpu's packed branch, starks_api.cu:1660-1676):
// the packed rows are unpacked straight into the column-major scratch, which the LDE then
// transforms in place.  col_bits: host array of nCols widths in 1..64; d_packed: N x
// words_per_row words with words_per_row = b200_packed_words_per_row(col_bits, nCols).
extern "C" int b200_commit_packed_device(uint64_t *root_host, uint64_t *d_lde, uint64_t *d_tree,
                                         const uint64_t *d_packed, uint64_t words_per_row, const uint32_t *col_bits,
                                         uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t arity,
                                         uint64_t *d_scratch, void *stream)
{
    int rc = check_shape(nBits, nBitsExt, nCols, arity);
    if (rc) return rc;
    if (nCols && !col_bits) return set_err(B200_EINVAL, "null column widths");
    for (uint64_t c = 0; c < nCols; c++)
        if (col_bits[c] < 1 || col_bits[c] > 64) return set_err(B200_EINVAL, "column width outside 1..64");
    if (nCols > unpack::COLS_MAX) return set_err(B200_EINVAL, "packed commit supports at most 12288 columns");
    if (nCols && words_per_row * 64 < unpack::packed_bits(col_bits, nCols))
        return set_err(B200_EINVAL, "words_per_row too small for the column widths");
    if ((rc = ensure_init_current())) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    if (!d_tree || (nCols && (!d_lde || !d_packed || !d_scratch))) return set_err(B200_EINVAL, "null buffer");
    if (nCols) {
        unpack::ColBytes cols;  // widths in the kernel parameters
        for (uint64_t c = 0; c < nCols; c++) cols.v[c] = (uint8_t)col_bits[c];
        {
            prof::Scope ps(prof::TRANSPOSE, s);
            CK(unpack::launch(d_scratch, d_packed, (const uint64_t *)nullptr, N, words_per_row, 0, 0, 0, cols, 0,
                              (uint32_t)nCols, s),
               "unpack");
            prof::count();
        }
        // the trace now sits column-major in the scratch; the LDE transforms it in place
        CK(ntt::lde(d_lde, d_scratch, false, (uint32_t)nBits, (uint32_t)nBitsExt, nCols, d_scratch, s), "lde");
    }
    CK(merkle::build_tree_arity(arity, d_tree, d_lde, 1, NExt, nCols, NExt, s, g_native_family.load()), "merkletree");
    if (root_host) {
        const uint64_t total = merkle::tree_num_elements(NExt, arity);
        CK(cudaMemcpyAsync(root_host, d_tree + total - 4, 32, cudaMemcpyDeviceToHost, s), "root D2H");
        CK(cudaStreamSynchronize(s), "sync");
    }
    return B200_OK;
}

// ------------------------------------------------------ streaming slot commit ----

// Widths -> the slot's width and bit-offset tables (host staging of 2 x 64 words).
static int stream_tables(uint64_t *tab, const uint64_t *colWidths, uint64_t nCols, uint64_t wordsPerRow)
{
    uint64_t off = 0;
    for (uint64_t c = 0; c < nCols; c++) {
        if (colWidths[c] < 1 || colWidths[c] > 64) return set_err(B200_EINVAL, "column width outside 1..64");
        tab[c] = colWidths[c];
        tab[stream::MAX_COLS + c] = off;
        off += colWidths[c];
    }
    if (off > 64 * wordsPerRow) return set_err(B200_EINVAL, "wordsPerRow too small for the column widths");
    return B200_OK;
}

// Indexed witness description for the host checks (col_source: 1 = table column).
struct IndexedDesc {
    const uint8_t *col_source;
    uint64_t index_bits;
    const uint64_t *d_table;
    uint64_t num_entries, words_per_entry;
};

// col_info[c] = width | source << 32, and the row / table bit budgets checked
static int indexed_info(uint64_t *info, const uint64_t *colWidths, uint64_t nCols, uint64_t wordsPerRow,
                        const IndexedDesc &ix)
{
    if (ix.index_bits > 64) return set_err(B200_EINVAL, "index header wider than 64 bits");
    uint64_t row_bits = ix.index_bits, tab_bits = 0;
    for (uint64_t c = 0; c < nCols; c++) {
        if (colWidths[c] < 1 || colWidths[c] > 64) return set_err(B200_EINVAL, "column width outside 1..64");
        const uint64_t src = ix.col_source[c] ? 1 : 0;
        info[c] = colWidths[c] | (src << 32);
        (src ? tab_bits : row_bits) += colWidths[c];
    }
    if (row_bits > 64 * wordsPerRow) return set_err(B200_EINVAL, "wordsPerRow too small for the row columns");
    if (tab_bits > 64 * ix.words_per_entry) return set_err(B200_EINVAL, "words_per_entry too small for the table columns");
    if (tab_bits && (!ix.d_table || ix.num_entries == 0)) return set_err(B200_EINVAL, "table columns without a table");
    return B200_OK;
}

// One streaming commit on a slot: H2D of the packed rows and the tables, the chunked LDE +
// absorb, the tree levels, the root D2H; synchronous.  ix: indexed witness, or null.
static int stream_commit_on(uint64_t *slot, uint64_t slot_words, cudaStream_t s, const void *h_packed,
                            uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t wordsPerRow,
                            const uint64_t *colWidths, uint64_t *root, int family, const IndexedDesc *ix = nullptr)
{
    if (nCols == 0 || nCols > stream::MAX_COLS || nBitsExt <= nBits || wordsPerRow == 0 || !colWidths || !h_packed ||
        !root)
        return set_err(B200_EINVAL, "streaming commit: nCols must be 1..64, nBitsExt > nBits, buffers non-null");
    int rc = check_shape(nBits, nBitsExt, nCols, 4);
    if (rc) return rc;
    const stream::Layout l = stream::layout(nBits, nBitsExt, wordsPerRow);
    if (l.total > slot_words) return set_err(B200_EINVAL, "slot too small for this shape");
    uint64_t tab[2 * stream::MAX_COLS] = {0};
    if (ix) {
        if (!ix->col_source) return set_err(B200_EINVAL, "null column sources");
        if ((rc = indexed_info(tab, colWidths, nCols, wordsPerRow, *ix))) return rc;
    } else if ((rc = stream_tables(tab, colWidths, nCols, wordsPerRow))) {
        return rc;
    }
    if ((rc = ensure_init_current())) return rc;
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    CK(cudaMemcpyAsync(slot + l.widths, tab, sizeof(tab), cudaMemcpyHostToDevice, s), "tables H2D");
    CK(cudaMemcpyAsync(slot + l.packed, h_packed, N * wordsPerRow * 8, cudaMemcpyHostToDevice, s), "packed H2D");
    stream::Indexed sx{};
    if (ix) sx = stream::Indexed{ix->d_table, ix->num_entries, ix->words_per_entry, ix->index_bits};
    const stream::Indexed *px = ix ? &sx : nullptr;
    CK(family == 1 ? stream::run<1>(slot, l, nBits, nBitsExt, nCols, wordsPerRow, s, px)
                   : stream::run<2>(slot, l, nBits, nBitsExt, nCols, wordsPerRow, s, px),
       "streaming commit");
    const uint64_t tsz = merkle::tree_num_elements(NExt, 4);
    CK(cudaMemcpyAsync(root, slot + l.tree + tsz - 4, 32, cudaMemcpyDeviceToHost, s), "root D2H");
    CK(cudaStreamSynchronize(s), "sync");
    return B200_OK;
}

extern "C" uint64_t stream_commit_slot_bytes(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t wordsPerRow)
{
    if (nCols == 0 || nCols > stream::MAX_COLS || nBitsExt <= nBits || wordsPerRow == 0 || nBitsExt > NTT_TWLG) return 0;
    return stream::layout(nBits, nBitsExt, wordsPerRow).total * 8;
}

extern "C" void configure_stream_commit_slots(void *d_buffers, uint64_t nSlots, uint64_t slotBytes)
{
    auto *b = (CommitBuffers *)d_buffers;
    if (!b) return;
    std::lock_guard<std::mutex> lk(b->mu);
    cudaSetDevice(b->device);
    for (cudaStream_t t : b->sc_streams) {
        cudaStreamSynchronize(t);
        cudaStreamDestroy(t);
    }
    b->sc_streams.clear();
    if (b->sc_base) cudaFree(b->sc_base);
    b->sc_base = nullptr;
    b->sc_slot_bytes = 0;
    if (nSlots == 0 || slotBytes == 0) return;
    slotBytes = (slotBytes + 255) & ~255ull;
    if (cudaMalloc((void **)&b->sc_base, nSlots * slotBytes) != cudaSuccess) {
        cudaGetLastError();
        b->sc_base = nullptr;
        b->error = set_err(B200_ENOMEM, "configure_stream_commit_slots: cudaMalloc");
        return;
    }
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);  // lo = numerically largest = lowest priority
    for (uint64_t i = 0; i < nSlots; i++) {
        cudaStream_t t;
        if (cudaStreamCreateWithPriority(&t, cudaStreamNonBlocking, lo) != cudaSuccess) {
            b->error = set_err(B200_ECUDA, "configure_stream_commit_slots: stream");
            return;
        }
        b->sc_streams.push_back(t);
    }
    b->sc_slot_bytes = slotBytes;
    b->sc_quiesced.store(0);
    g_stream_buffers.store(b);
}

extern "C" uint64_t get_stream_commit_slots(void *d_buffers)
{
    auto *b = (CommitBuffers *)d_buffers;
    return b ? b->sc_streams.size() : 0;
}

// The reference carves its slots out of its unified buffer and reports where they start; this
// library allocates them on their own, so the offset within that allocation is 0.
extern "C" uint64_t get_stream_commit_floor(void *d_buffers)
{
    auto *b = (CommitBuffers *)d_buffers;
    if (!b) return UINT64_MAX;
    return 0;
}

// Return codes follow commit_witness_streaming (api/starks_api.cu:2290-2348): 0 ok, -11 no slots,
// -12 slot index out of range, -13 slot too small for the shape, -14 quiesced by
// stream_commit_pause, -15 hash family is not Poseidon1; -10 invalid shape or widths.  The
// indexed (instruction-table) witness is not supported (-16).
extern "C" int64_t commit_witness_streaming(void *d_buffers, uint64_t slotIdx, uint64_t airgroupId, uint64_t airId,
                                            void *packed, uint64_t nBits, uint64_t nBitsExt, uint64_t nCols,
                                            uint64_t wordsPerRow, void *colWidths, void *root)
{
    auto *b = (CommitBuffers *)d_buffers;
    if (!b || b->sc_streams.empty()) return -11;
    if (slotIdx >= b->sc_streams.size()) return -12;
    if (g_hash_family.load() != 1) return -15;
    if (stream_commit_slot_bytes(nBits, nBitsExt, nCols, wordsPerRow) == 0) return -10;
    if (stream::layout(nBits, nBitsExt, wordsPerRow).total * 8 > b->sc_slot_bytes) return -13;
    if (b->sc_quiesced.load()) return -14;
    b->sc_inflight++;
    if (b->sc_quiesced.load()) {
        b->sc_inflight--;
        return -14;
    }
    cudaSetDevice(b->device);
    IndexedDesc ixd{};
    const IndexedDesc *ix = nullptr;
    {
        std::lock_guard<std::mutex> lk(b->mu);
        auto it = b->indexed.find({airgroupId, airId});
        if (it != b->indexed.end()) {
            if (!it->second.d_table) {
                b->sc_inflight--;
                set_err(B200_EINVAL, "indexed air without a registered instruction table");
                return -16;
            }
            if (it->second.col_source.size() != nCols) {
                b->sc_inflight--;
                set_err(B200_EINVAL, "indexed air registered with another column count");
                return -10;
            }
            ixd = IndexedDesc{it->second.col_source.data(), it->second.index_bits, it->second.d_table,
                              it->second.num_entries, it->second.words_per_entry};
            ix = &ixd;
        }
    }
    uint64_t *slot = b->sc_base + slotIdx * (b->sc_slot_bytes / 8);
    int rc = stream_commit_on(slot, b->sc_slot_bytes / 8, b->sc_streams[slotIdx], packed, nBits, nBitsExt, nCols,
                              wordsPerRow, (const uint64_t *)colWidths, (uint64_t *)root, 1, ix);
    b->sc_inflight--;
    return rc == B200_OK ? 0 : -10;
}

// Reject new slot commits and wait (bounded, about 2 s) for the running ones to finish.

extern "C" void stream_commit_pause(void)
{
    CommitBuffers *b = g_stream_buffers.load();
    if (!b) return;
    b->sc_quiesced.store(1);
    for (int i = 0; i < 4000 && b->sc_inflight.load() != 0; i++) std::this_thread::sleep_for(std::chrono::microseconds(500));
}

// Native form with caller-owned device slot memory and the native hash family (no reference
// counterpart; the reference entry above is Poseidon1-only and owns its slots).
extern "C" int b200_stream_commit_packed(uint64_t *d_slot, uint64_t slot_words, const uint64_t *h_packed,
                                         uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t wordsPerRow,
                                         const uint64_t *colWidths, uint64_t *root, void *stream)
{
    if (!d_slot) return set_err(B200_EINVAL, "null slot");
    return stream_commit_on(d_slot, slot_words, (cudaStream_t)stream, h_packed, nBits, nBitsExt, nCols, wordsPerRow,
                            colWidths, root, g_native_family.load());
}

// ------------------------------------------------------------ indexed witness ----
// Stands in for the setup's PackedInfo of an indexed AIR: which columns come from the
// instruction table (col_source[c] = 1) and the width of the row's leading index.
extern "C" int b200_register_indexed_air(void *d_buffers, uint64_t airgroupId, uint64_t airId, uint64_t nCols,
                                         const uint8_t *col_source, uint64_t index_bits)
{
    auto *b = (CommitBuffers *)d_buffers;
    if (!b || (nCols && !col_source)) return set_err(B200_EINVAL, "null argument");
    if (index_bits > 64) return set_err(B200_EINVAL, "index header wider than 64 bits");
    std::lock_guard<std::mutex> lk(b->mu);
    auto &a = b->indexed[{airgroupId, airId}];
    a.col_source.assign(col_source, col_source + nCols);
    a.index_bits = index_bits;
    return B200_OK;
}

// register_instruction_table (starks_api.hpp:192): the AIR's instruction table, num_entries
// entries of words_per_entry words (host), copied to the device and kept with the buffers.
extern "C" void register_instruction_table(void *d_buffers, uint64_t airgroupId, uint64_t airId, uint64_t *table,
                                           uint64_t num_entries, uint64_t words_per_entry)
{
    auto *b = (CommitBuffers *)d_buffers;
    if (!b || !table || num_entries == 0) {
        set_err(B200_EINVAL, "register_instruction_table: empty table");
        if (b) b->error = B200_EINVAL;
        return;
    }
    std::lock_guard<std::mutex> lk(b->mu);
    cudaSetDevice(b->device);
    auto &a = b->indexed[{airgroupId, airId}];
    if (a.d_table) cudaFree(a.d_table);
    a.d_table = nullptr;
    const uint64_t words = num_entries * (words_per_entry ? words_per_entry : 1);
    if (cudaMalloc((void **)&a.d_table, words * 8) != cudaSuccess ||
        cudaMemcpy(a.d_table, table, num_entries * words_per_entry * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        if (a.d_table) cudaFree(a.d_table);
        a.d_table = nullptr;
        b->error = set_err(B200_ENOMEM, "register_instruction_table: device copy");
        return;
    }
    a.num_entries = num_entries;
    a.words_per_entry = words_per_entry;
}

// Native commit of an indexed witness (device rows and table; col_bits, col_source on the host):
// the reference's unpack_indexed (starks_gpu.cu:125-185) straight into the column-major scratch,
// then the LDE in place and the tree, like b200_commit_packed_device.
extern "C" int b200_commit_indexed_device(uint64_t *root_host, uint64_t *d_lde, uint64_t *d_tree,
                                          const uint64_t *d_rows, uint64_t words_per_row, const uint64_t *d_table,
                                          uint64_t num_entries, uint64_t words_per_entry, uint64_t index_bits,
                                          const uint64_t *col_bits, const uint8_t *col_source, uint64_t nBits,
                                          uint64_t nBitsExt, uint64_t nCols, uint64_t arity, uint64_t *d_scratch,
                                          void *stream)
{
    int rc = check_shape(nBits, nBitsExt, nCols, arity);
    if (rc) return rc;
    if (nCols && (!col_bits || !col_source)) return set_err(B200_EINVAL, "null column description");
    if (nCols > unpack::COLS_MAX) return set_err(B200_EINVAL, "indexed commit supports at most 12288 columns");
    std::vector<uint64_t> info(nCols);
    const IndexedDesc ix{col_source, index_bits, d_table, num_entries, words_per_entry};
    if (nCols && (rc = indexed_info(info.data(), col_bits, nCols, words_per_row, ix))) return rc;
    if ((rc = ensure_init_current())) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    if (!d_tree || (nCols && (!d_lde || !d_rows || !d_scratch))) return set_err(B200_EINVAL, "null buffer");
    if (nCols) {
        unpack::ColBytes cols;  // width | table source << 7 per column, in the kernel parameters
        for (uint64_t c = 0; c < nCols; c++) cols.v[c] = (uint8_t)((info[c] & 127) | ((info[c] >> 32) << 7));
        {
            prof::Scope ps(prof::TRANSPOSE, s);
            CK(unpack::launch(d_scratch, d_rows, d_table, N, words_per_row, words_per_entry, num_entries,
                              (uint32_t)index_bits, cols, 0, (uint32_t)nCols, s),
               "indexed unpack");
            prof::count();
        }
        CK(ntt::lde(d_lde, d_scratch, false, (uint32_t)nBits, (uint32_t)nBitsExt, nCols, d_scratch, s), "lde");
    }
    CK(merkle::build_tree_arity(arity, d_tree, d_lde, 1, NExt, nCols, NExt, s, g_native_family.load()), "merkletree");
    if (root_host) {
        const uint64_t total = merkle::tree_num_elements(NExt, arity);
        CK(cudaMemcpyAsync(root_host, d_tree + total - 4, 32, cudaMemcpyDeviceToHost, s), "root D2H");
        CK(cudaStreamSynchronize(s), "sync");
    }
    return B200_OK;
}

// Native streaming commit of an indexed witness (host rows, device table).
extern "C" int b200_stream_commit_indexed(uint64_t *d_slot, uint64_t slot_words, const uint64_t *h_rows,
                                          uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t words_per_row,
                                          const uint64_t *col_bits, const uint8_t *col_source, uint64_t index_bits,
                                          const uint64_t *d_table, uint64_t num_entries, uint64_t words_per_entry,
                                          uint64_t *root, void *stream)
{
    if (!d_slot) return set_err(B200_EINVAL, "null slot");
    const IndexedDesc ix{col_source, index_bits, d_table, num_entries, words_per_entry};
    return stream_commit_on(d_slot, slot_words, (cudaStream_t)stream, h_rows, nBits, nBitsExt, nCols, words_per_row,
                            col_bits, root, g_native_family.load(), &ix);
}

// ------------------------------------------------ tree level and digest reduction ----
// MerkleTreeGL::getLevel (merkleTreeGL.cpp:84-101): with last_level_verification = llv > 0, the
// first level holding <= arity^llv nodes, copied to d_out and zero-filled to arity^llv nodes
// (4 words each) — the level that openings of that depth are checked against.
extern "C" uint64_t b200_tree_last_level_words(uint64_t arity, uint64_t last_level_verification)
{
    uint64_t n = 1;
    for (uint64_t i = 0; i < last_level_verification; i++) n *= arity;
    return 4 * n;
}

extern "C" int b200_tree_last_level_device(uint64_t *d_out, const uint64_t *d_tree, uint64_t NExt, uint64_t arity,
                                           uint64_t last_level_verification, void *stream)
{
    if (arity < 2 || arity > 4 || last_level_verification == 0 || last_level_verification > 32)
        return set_err(B200_EINVAL, "arity 2..4 and last_level_verification >= 1 required");
    if (!d_out || !d_tree) return set_err(B200_EINVAL, "null buffer");
    const uint64_t stop = b200_tree_last_level_words(arity, last_level_verification) / 4;
    uint64_t n = NExt, offset = 0;
    while (n > stop) {
        n = (n + arity - 1) / arity;
        offset += n * arity * 4;
    }
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaMemcpyAsync(d_out, d_tree + offset, n * 4 * 8, cudaMemcpyDeviceToDevice, s), "level copy");
    if (stop > n) CK(cudaMemsetAsync(d_out + n * 4, 0, (stop - n) * 4 * 8, s), "level zero fill");
    return B200_OK;
}

// merkletreeReduce (poseidon2_goldilocks.hpp merkletreeReduce; W = 4 * arity): the tree levels
// above n given digests (d_digests, 4 words each), in d_tree (b200_tree_num_elements(n, arity)
// words, level 0 = a copy of the digests), with the native hash family; the root to root_host.
extern "C" int b200_merkletree_reduce_device(uint64_t *root_host, const uint64_t *d_digests, uint64_t n,
                                             uint64_t arity, uint64_t *d_tree, void *stream)
{
    if (arity < 2 || arity > 4) return set_err(B200_EINVAL, "arity must be 2, 3 or 4");
    if (n == 0 || !d_digests || !d_tree) return set_err(B200_EINVAL, "empty digest list or null buffer");
    int rc = ensure_init_current();
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaMemcpyAsync(d_tree, d_digests, n * 4 * 8, cudaMemcpyDeviceToDevice, s), "digests copy");
    const int fam = g_native_family.load();
    cudaError_t e;
    switch (arity) {
    case 2: e = fam == 1 ? merkle::build_levels<8, 1>(d_tree, n, s) : merkle::build_levels<8, 2>(d_tree, n, s); break;
    case 3: e = fam == 1 ? merkle::build_levels<12, 1>(d_tree, n, s) : merkle::build_levels<12, 2>(d_tree, n, s); break;
    default: e = fam == 1 ? merkle::build_levels<16, 1>(d_tree, n, s) : merkle::build_levels<16, 2>(d_tree, n, s); break;
    }
    CK(e, "tree levels");
    if (root_host) {
        const uint64_t total = merkle::tree_num_elements(n, arity);
        CK(cudaMemcpyAsync(root_host, d_tree + total - 4, 32, cudaMemcpyDeviceToHost, s), "root D2H");
        CK(cudaStreamSynchronize(s), "sync");
    }
    return B200_OK;
}
