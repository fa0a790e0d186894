// Row sponge ("linear hash") and arity-k Merkle tree levels, Poseidon2 or Poseidon1.
//
// Semantics follow the reference CPU path bit for bit:
//   linear hash  poseidon2_goldilocks.cpp:42-77 — capacity zeroed at the start; every
//                block overwrites words [0, n) with input, zero-fills [n, RATE) and carries
//                the previous output words [0, 4) into the capacity; no length padding;
//                0 columns give the zero digest.
//   tree         poseidon2_goldilocks.cpp:129-175 — digests of a level are contiguous
//                4-word groups; (arity - pending % arity) % arity zero digests pad the level
//                inside the buffer; parent i is the first 4 words of the permutation of the
//                W = 4*arity words of its children; the root is the last 4 words
//                (goldilocks_tooling.hpp:9-21 gives the buffer size).
//
// Layout: the extended trace is addressed as element (row, col) = src[row*rs + col*cs], so
// the same kernel reads the column-major device LDE (rs = 1, cs = nrows; warp loads are
// 256 B contiguous) or a row-major buffer (rs = ncols, cs = 1).
#pragma once
#include "coop.cuh"
#include "poseidon1.cuh"
#include "poseidon2.cuh"
#include "prof.cuh"

namespace merkle {

constexpr int TPB = 128;  // threads per CTA of the hashing kernels (one row / node / state each)

// Hash family (the reference's set_hash_family): 1 = Poseidon1, 2 = Poseidon2.  Both use the same
// sponge and tree; the Poseidon1 permutation needs a second W x TPB shared area for its matrix
// steps, right after the state area.
template <int FAM>
struct Family {
    static constexpr int SMEM_AREAS = FAM == 1 ? 2 : 1;
    // resident CTAs per SM the register budget must allow (registers <= 64 K / (MIN_CTAS * 128)):
    // Poseidon1's 32 KB of shared memory per CTA fits 7 CTAs, so its registers are capped to
    // match (72); Poseidon2 keeps 12 resident CTAs (<= 42 registers, the 40 it needs)
    static constexpr int MIN_CTAS = FAM == 1 ? 7 : 12;
};

template <int W, int FAM>
__device__ __forceinline__ void permute_fam(uint64_t *st)
{
    if constexpr (FAM == 1)
        p1::permute_smem<W, TPB>(st, st + W * TPB);
    else
        p2::permute_smem<W, TPB>(st);
}

// Digest i of a level sits at base + 4*i words, so every digest has the base's alignment.  A
// 16-byte aligned base takes two 16-byte stores / loads per digest, any other base (a tree at an odd
// word offset of a caller's buffer) four 8-byte ones; the test is uniform across the launch.
__device__ __forceinline__ void store_digest(uint64_t *d, const uint64_t *st)
{
    const uint64_t a = gl::canon(st[0]), b = gl::canon(st[TPB]), c = gl::canon(st[2 * TPB]), e = gl::canon(st[3 * TPB]);
    if ((reinterpret_cast<uintptr_t>(d) & 15) == 0) {
        reinterpret_cast<ulonglong2 *>(d)[0] = make_ulonglong2(a, b);
        reinterpret_cast<ulonglong2 *>(d)[1] = make_ulonglong2(c, e);
    } else {
        d[0] = a;
        d[1] = b;
        d[2] = c;
        d[3] = e;
    }
}

// Sponge of one row; st = this thread's state slot in a W x TPB shared array.
template <int W, int FAM = 2>
__device__ __forceinline__ void leaf_row(uint64_t *st, uint64_t *__restrict__ digests,
                                         const uint64_t *__restrict__ src, uint64_t rs, uint64_t cs, uint64_t ncols,
                                         uint64_t row)
{
    constexpr int RATE = W - 4;
#pragma unroll
    for (int i = 0; i < W; i++) st[i * TPB] = 0;
    const uint64_t *p = src + row * rs;
    for (uint64_t done = 0; done < ncols; done += RATE) {
        const uint64_t n = ncols - done;
        if (done != 0) {
#pragma unroll
            for (int j = 0; j < 4; j++) st[(RATE + j) * TPB] = st[j * TPB];
        }
        if (n >= (uint64_t)RATE) {
#pragma unroll
            for (int i = 0; i < RATE; i++) st[i * TPB] = __ldg(p + (done + i) * cs);
        } else {
#pragma unroll
            for (int i = 0; i < RATE; i++) st[i * TPB] = (uint64_t)i < n ? __ldg(p + (done + i) * cs) : 0ull;
        }
        permute_fam<W, FAM>(st);
    }
    // ncols == 0 leaves the state zeroed: the zero digest
    store_digest(digests + row * 4, st);
}

template <int W, int FAM = 2>
__global__ void __launch_bounds__(TPB, Family<FAM>::MIN_CTAS) leaf_hash_kernel(uint64_t *__restrict__ digests,
                                                        const uint64_t *__restrict__ src, uint64_t rs,
                                                        uint64_t cs, uint64_t ncols, uint64_t nrows)
{
    __shared__ uint64_t sm[Family<FAM>::SMEM_AREAS * W * TPB];
    const uint64_t row = (uint64_t)blockIdx.x * TPB + threadIdx.x;
    if (row < nrows) leaf_row<W, FAM>(sm + threadIdx.x, digests, src, rs, cs, ncols, row);
}

// Parent i of one tree level: `pending` child digests at `level`, `pad` zero digests written
// after them (by the last parent), parents written to `out` (= level + 4*(pending + pad)).
template <int W, int FAM = 2>
__device__ __forceinline__ void node_one(uint64_t *st, uint64_t *__restrict__ level, uint64_t pending, uint64_t pad,
                                         uint64_t parents, uint64_t *__restrict__ out, uint64_t i)
{
    constexpr int ARITY = W / 4;
#pragma unroll
    for (int c = 0; c < ARITY; c++) {
        const uint64_t child = i * ARITY + c;
        if (child < pending) {
            const uint64_t *q = level + child * 4;
            if ((reinterpret_cast<uintptr_t>(q) & 15) == 0) {
                const ulonglong2 v0 = reinterpret_cast<const ulonglong2 *>(q)[0],
                                 v1 = reinterpret_cast<const ulonglong2 *>(q)[1];
                st[(4 * c + 0) * TPB] = v0.x;
                st[(4 * c + 1) * TPB] = v0.y;
                st[(4 * c + 2) * TPB] = v1.x;
                st[(4 * c + 3) * TPB] = v1.y;
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) st[(4 * c + j) * TPB] = q[j];
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) st[(4 * c + j) * TPB] = 0;
        }
    }
    if (i == parents - 1) {
        for (uint64_t z = 0; z < pad * 4; z++) level[pending * 4 + z] = 0;
    }
    permute_fam<W, FAM>(st);
    store_digest(out + i * 4, st);
}

template <int W, int FAM = 2>
__global__ void __launch_bounds__(TPB, Family<FAM>::MIN_CTAS) node_kernel(uint64_t *__restrict__ level, uint64_t pending, uint64_t pad,
                                                   uint64_t parents, uint64_t *__restrict__ out)
{
    __shared__ uint64_t sm[Family<FAM>::SMEM_AREAS * W * TPB];
    const uint64_t i = (uint64_t)blockIdx.x * TPB + threadIdx.x;
    if (i < parents) node_one<W, FAM>(sm + threadIdx.x, level, pending, pad, parents, out, i);
}

// Whole permutations of n independent states (permute / permuteTrunc checks).
template <int W, int FAM = 2>
__global__ void __launch_bounds__(TPB, Family<FAM>::MIN_CTAS) permute_kernel(uint64_t *__restrict__ out, const uint64_t *__restrict__ in,
                                                      uint64_t n)
{
    __shared__ uint64_t sm[Family<FAM>::SMEM_AREAS * W * TPB];
    uint64_t *st = sm + threadIdx.x;
    const uint64_t i = (uint64_t)blockIdx.x * TPB + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int j = 0; j < W; j++) st[j * TPB] = in[i * W + j];
    permute_fam<W, FAM>(st);
#pragma unroll
    for (int j = 0; j < W; j++) out[i * W + j] = gl::canon(st[j * TPB]);
}

inline uint64_t tree_num_elements(uint64_t nrows, uint64_t arity)
{
    uint64_t total = nrows, level = nrows;
    while (level > 1) {
        total += (arity - level % arity) % arity;
        level = (level + arity - 1) / arity;
        total += level;
    }
    return total * 4;
}

// Below this many states per launch the one-thread-per-state hashing kernels leave the GPU idle
// and take the latency of one whole permutation per thread (~40 us for Poseidon2 W16); the
// cooperative kernels (coop.cuh, one state per 16 lanes) take it instead.
constexpr uint64_t COOP_MAX_STATES = 8192;

// Every tree level above `nrows` leaf digests already at the start of d_tree, on `stream`.
// Levels of more than COOP_MAX_STATES parents one thread per parent, smaller ones cooperatively,
// and the last levels (<= coop::TAIL_THREADS / G parents) in one launch; both hash families.
template <int W, int FAM = 2>
cudaError_t build_levels(uint64_t *d_tree, uint64_t nrows, cudaStream_t stream)
{
    constexpr uint64_t ARITY = W / 4;
    const unsigned tpb = TPB;
    prof::Scope ps(prof::TREE_LEVELS, stream);
    uint64_t pending = nrows, base = 0;
    while (pending > 1) {
        const uint64_t pad = (ARITY - pending % ARITY) % ARITY;
        const uint64_t parents = (pending + ARITY - 1) / ARITY;
        uint64_t *lvl = d_tree + base;
        {
            constexpr uint64_t G = coop::Tab<W>::G;
            if (parents <= (uint64_t)coop::TAIL_THREADS / G) {
                coop::tree_tail_kernel<W, FAM><<<1, coop::TAIL_THREADS, 0, stream>>>(lvl, pending);
                prof::count();
                break;
            }
            if (parents <= COOP_MAX_STATES) {
                const uint64_t threads = parents * G;
                coop::node_coop_kernel<W, FAM>
                    <<<(unsigned)((threads + coop::CTA_THREADS - 1) / coop::CTA_THREADS), coop::CTA_THREADS, 0,
                       stream>>>(lvl, pending, pad, parents, lvl + (pending + pad) * 4);
                prof::count();
                base += (pending + pad) * 4;
                pending = parents;
                continue;
            }
        }
        node_kernel<W, FAM><<<(unsigned)((parents + tpb - 1) / tpb), tpb, 0, stream>>>(lvl, pending, pad, parents,
                                                                                   lvl + (pending + pad) * 4);
        prof::count();
        base += (pending + pad) * 4;
        pending = parents;
    }
    return cudaGetLastError();
}

// Leaf digests and every level up to the root, on `stream`.
template <int W, int FAM = 2>
cudaError_t build_tree(uint64_t *d_tree, const uint64_t *d_src, uint64_t rs, uint64_t cs, uint64_t ncols,
                       uint64_t nrows, cudaStream_t stream)
{
    if (nrows == 0) return cudaSuccess;
    const unsigned tpb = TPB;
    {
        prof::Scope ps(prof::LEAF_HASH, stream);
        if (nrows <= COOP_MAX_STATES) {
            const uint64_t threads = nrows * coop::Tab<W>::G;
            coop::leaf_coop_kernel<W, FAM><<<(unsigned)((threads + coop::CTA_THREADS - 1) / coop::CTA_THREADS),
                                             coop::CTA_THREADS, 0, stream>>>(d_tree, d_src, rs, cs, ncols, nrows);
        } else {
            leaf_hash_kernel<W, FAM><<<(unsigned)((nrows + tpb - 1) / tpb), tpb, 0, stream>>>(d_tree, d_src, rs, cs,
                                                                                           ncols, nrows);
        }
        prof::count();
    }
    return build_levels<W, FAM>(d_tree, nrows, stream);
}

// family: 1 = Poseidon1, otherwise Poseidon2; W = 4 * arity (MerkleTreeGL::merkelize)
inline cudaError_t build_tree_arity(uint64_t arity, uint64_t *d_tree, const uint64_t *d_src, uint64_t rs,
                                    uint64_t cs, uint64_t ncols, uint64_t nrows, cudaStream_t stream, int family = 2)
{
    if (family == 1) {
        switch (arity) {
        case 2: return build_tree<8, 1>(d_tree, d_src, rs, cs, ncols, nrows, stream);
        case 3: return build_tree<12, 1>(d_tree, d_src, rs, cs, ncols, nrows, stream);
        case 4: return build_tree<16, 1>(d_tree, d_src, rs, cs, ncols, nrows, stream);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (arity) {
    case 2: return build_tree<8>(d_tree, d_src, rs, cs, ncols, nrows, stream);
    case 3: return build_tree<12>(d_tree, d_src, rs, cs, ncols, nrows, stream);
    case 4: return build_tree<16>(d_tree, d_src, rs, cs, ncols, nrows, stream);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace merkle
