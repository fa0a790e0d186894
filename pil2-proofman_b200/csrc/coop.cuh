// Cooperative Poseidon2 and Poseidon1 for work too small to fill the GPU with one thread per
// state: the top levels of a tree and the leaves of tiny instances.
//
// One state per group of G lanes of a warp (G = 16 for W = 12 and 16, G = 8 for W = 8);
// lane k of the group holds word k (lanes k >= W hold zero).  The S-boxes of a full round
// run on all lanes at once; M_E takes a lane's block of four words by shuffles, applies its
// row of M4 (small coefficients, two 64-bit sums of 32x32 products) and adds the column sum
// over the blocks (xor shuffles over the block bits); the partial-round sum is an xor-shuffle
// reduction over the group that runs beside x0's S-box.  A permutation then costs the latency
// of about 30 S-box chains instead of 952 dependent multiplications: ~5x less time for a
// state, at several times the instructions per state, so it is used only where the
// one-thread-per-state kernels leave the GPU idle.  The arithmetic is the same modular
// arithmetic as poseidon2.cuh (loose words, 96-bit accumulators), so the canonical results are
// identical.
#pragma once
#include "gl64.cuh"
#include "poseidon1.cuh"
#include "poseidon2_constants.h"

// Round constants and diagonals in global memory: lanes read different entries, which the
// constant cache would serialise.
__device__ uint64_t g_coop_C8[P2_NC_8] = {P2_C8_LIST};
__device__ uint64_t g_coop_D8[8] = {P2_D8_LIST};
__device__ uint64_t g_coop_C12[P2_NC_12] = {P2_C12_LIST};
__device__ uint64_t g_coop_D12[12] = {P2_D12_LIST};
__device__ uint64_t g_coop_C16[P2_NC_16] = {P2_C16_LIST};
__device__ uint64_t g_coop_D16[16] = {P2_D16_LIST};
// Poseidon1 (hash family 1): round constants C, small MDS M, pre-partial matrix P, sparse S
__device__ uint64_t g_coop1_C8[P1_NC_8] = {P1_C8_LIST};
__device__ uint64_t g_coop1_M8[64] = {P1_M8_LIST};
__device__ uint64_t g_coop1_P8[64] = {P1_P8_LIST};
__device__ uint64_t g_coop1_S8[P1_NS_8] = {P1_S8_LIST};
__device__ uint64_t g_coop1_C12[P1_NC_12] = {P1_C12_LIST};
__device__ uint64_t g_coop1_M12[144] = {P1_M12_LIST};
__device__ uint64_t g_coop1_P12[144] = {P1_P12_LIST};
__device__ uint64_t g_coop1_S12[P1_NS_12] = {P1_S12_LIST};
__device__ uint64_t g_coop1_C16[P1_NC_16] = {P1_C16_LIST};
__device__ uint64_t g_coop1_M16[256] = {P1_M16_LIST};
__device__ uint64_t g_coop1_P16[256] = {P1_P16_LIST};
__device__ uint64_t g_coop1_S16[P1_NS_16] = {P1_S16_LIST};

namespace coop {

constexpr int NPARTIAL = 22;

template <int W>
struct Tab;
template <>
struct Tab<8> {
    static constexpr int G = 8;
    static __device__ __forceinline__ const uint64_t *C() { return g_coop_C8; }
    static __device__ __forceinline__ const uint64_t *D() { return g_coop_D8; }
};
template <>
struct Tab<12> {
    static constexpr int G = 16;
    static __device__ __forceinline__ const uint64_t *C() { return g_coop_C12; }
    static __device__ __forceinline__ const uint64_t *D() { return g_coop_D12; }
};
template <>
struct Tab<16> {
    static constexpr int G = 16;
    static __device__ __forceinline__ const uint64_t *C() { return g_coop_C16; }
    static __device__ __forceinline__ const uint64_t *D() { return g_coop_D16; }
};

template <int W>
struct Tab1;
template <>
struct Tab1<8> {
    static __device__ __forceinline__ const uint64_t *C() { return g_coop1_C8; }
    static __device__ __forceinline__ const uint64_t *M() { return g_coop1_M8; }
    static __device__ __forceinline__ const uint64_t *P() { return g_coop1_P8; }
    static __device__ __forceinline__ const uint64_t *S() { return g_coop1_S8; }
};
template <>
struct Tab1<12> {
    static __device__ __forceinline__ const uint64_t *C() { return g_coop1_C12; }
    static __device__ __forceinline__ const uint64_t *M() { return g_coop1_M12; }
    static __device__ __forceinline__ const uint64_t *P() { return g_coop1_P12; }
    static __device__ __forceinline__ const uint64_t *S() { return g_coop1_S12; }
};
template <>
struct Tab1<16> {
    static __device__ __forceinline__ const uint64_t *C() { return g_coop1_C16; }
    static __device__ __forceinline__ const uint64_t *M() { return g_coop1_M16; }
    static __device__ __forceinline__ const uint64_t *P() { return g_coop1_P16; }
    static __device__ __forceinline__ const uint64_t *S() { return g_coop1_S16; }
};

__device__ __forceinline__ uint64_t shfl_u64(uint64_t x, int src)
{
    const uint32_t lo = __shfl_sync(0xffffffffu, gl::lo32(x), src);
    const uint32_t hi = __shfl_sync(0xffffffffu, gl::hi32(x), src);
    return gl::mk64(lo, hi);
}

// the three low 32-bit words of an accumulator (values < 2^96)
__device__ __forceinline__ gl::Acc shfl_xor_acc(gl::Acc a, int m)
{
    const uint32_t w0 = __shfl_xor_sync(0xffffffffu, (uint32_t)a.v, m);
    const uint32_t w1 = __shfl_xor_sync(0xffffffffu, (uint32_t)(a.v >> 32), m);
    const uint32_t w2 = __shfl_xor_sync(0xffffffffu, (uint32_t)(a.v >> 64), m);
    return gl::Acc{((unsigned __int128)w2 << 64) | ((unsigned __int128)w1 << 32) | w0};
}

// sum of a over the lanes that differ from this one only in lane bits [LO_BIT, HI_BIT) (xor
// butterfly; every lane ends with the sum)
template <int LO_BIT, int HI_BIT>
__device__ __forceinline__ gl::Acc xor_sum(gl::Acc a)
{
#pragma unroll
    for (int b = LO_BIT; b < HI_BIT; b++) a = gl::acc_add(a, shfl_xor_acc(a, 1 << b));
    return a;
}

// Row j of M4 = [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]] as four small coefficients.
struct Row {
    uint32_t m0, m1, m2, m3;
};
__device__ __forceinline__ Row m4_row(int j)
{
    // packed by column: byte j of each word
    const uint32_t c0 = 0x01010405u, c1 = 0x01030607u, c2 = 0x04050101u, c3 = 0x06070103u;
    const int sh = 8 * j;
    return Row{(c0 >> sh) & 0xffu, (c1 >> sh) & 0xffu, (c2 >> sh) & 0xffu, (c3 >> sh) & 0xffu};
}

// sum_i m_i * a_i for loose a_i and small m_i, as a 96-bit accumulator (two 64-bit sums of 32x32
// products over the low and high halves)
__device__ __forceinline__ gl::Acc dot4(const Row &m, uint64_t a0, uint64_t a1, uint64_t a2, uint64_t a3)
{
    uint64_t L, H;
    asm("mul.wide.u32 %0, %1, %2;" : "=l"(L) : "r"(gl::lo32(a0)), "r"(m.m0));
    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(L) : "r"(gl::lo32(a1)), "r"(m.m1));
    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(L) : "r"(gl::lo32(a2)), "r"(m.m2));
    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(L) : "r"(gl::lo32(a3)), "r"(m.m3));
    asm("mul.wide.u32 %0, %1, %2;" : "=l"(H) : "r"(gl::hi32(a0)), "r"(m.m0));
    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(H) : "r"(gl::hi32(a1)), "r"(m.m1));
    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(H) : "r"(gl::hi32(a2)), "r"(m.m2));
    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(H) : "r"(gl::hi32(a3)), "r"(m.m3));
    return gl::acc_lohi(L, H);  // L, H < 2^37
}

// M_E on the group's state: lane k (block k/4, row k%4) gets M4(block)_k%4 + sum over the blocks
// of M4(block)_k%4.  `live` = this lane holds a word (k < W); other lanes contribute nothing.
template <int W>
__device__ __forceinline__ uint64_t external_layer(uint64_t x, int gbase, int k, bool live, const Row &row)
{
    constexpr int G = Tab<W>::G;
    const int b0 = gbase + (k & ~3);
    const uint64_t a0 = shfl_u64(x, b0), a1 = shfl_u64(x, b0 + 1), a2 = shfl_u64(x, b0 + 2), a3 = shfl_u64(x, b0 + 3);
    gl::Acc y = dot4(row, a0, a1, a2, a3);
    if (!live) y = gl::Acc{0};
    const gl::Acc t = xor_sum<2, (G == 16 ? 4 : 3)>(y);
    return gl::acc_reduce(gl::acc_add(y, t));
}

// The permutation of the group's state (lane k: word k, loose in, loose out; zero for k >= W).
// gbase: first lane of the group within the warp.  All 32 lanes of the warp must call it.
template <int W>
__device__ __forceinline__ uint64_t permute(uint64_t x, int gbase, int k)
{
    constexpr int G = Tab<W>::G;
    const bool live = k < W;
    const int kk = live ? k : 0;
    const uint64_t *C = Tab<W>::C();
    const Row row = m4_row(k & 3);
    const uint64_t d = __ldg(Tab<W>::D() + kk);
    if (!live) x = 0;
    x = external_layer<W>(x, gbase, k, live, row);
#pragma unroll 1
    for (int r = 0; r < 8; r++) {
        const uint64_t c = __ldg(C + (r < 4 ? r * W : 4 * W + NPARTIAL + (r - 4) * W) + kk);
        x = gl::pow7(gl::add_c(x, c));
        x = external_layer<W>(x, gbase, k, live, row);
        if (r == 3) {
#pragma unroll 1
            for (int pr = 0; pr < NPARTIAL; pr++) {
                // sum of x_1.. (beside the S-box of x0, which every lane computes on its own word)
                gl::Acc rest = gl::acc((live && k != 0) ? x : 0ull);
                rest = xor_sum<0, (G == 16 ? 4 : 3)>(rest);
                const uint64_t s0 = gl::pow7(gl::add_c(x, __ldg(C + 4 * W + pr)));
                const uint64_t x0 = shfl_u64(s0, gbase);
                const uint64_t sum = gl::acc_reduce(gl::acc_add64(rest, x0));
                x = gl::mul_add(k == 0 ? x0 : x, d, sum);
                if (!live) x = 0;
            }
        }
    }
    return x;
}

// Poseidon1 matrix steps for lane k: out_k = sum_j mat[j][k] x_j over the group's words (gathered
// by shuffles).  The small-entry M as two 64-bit sums of 32x32 products; the full-entry P in
// 160 bits (p1::Acc160).
template <int W>
__device__ __forceinline__ uint64_t mvp_small1(uint64_t x, int gbase, int kk)
{
    const uint64_t *M = Tab1<W>::M();
    uint64_t L = 0, H = 0;
#pragma unroll
    for (int j = 0; j < W; j++) {
        const uint64_t xj = shfl_u64(x, gbase + j);
        const uint32_t m = (uint32_t)__ldg(M + j * W + kk);
        asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(L) : "r"(gl::lo32(xj)), "r"(m));
        asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(H) : "r"(gl::hi32(xj)), "r"(m));
    }
    return gl::acc_reduce(gl::acc_lohi(L, H));
}

template <int W>
__device__ __forceinline__ uint64_t mvp_full1(uint64_t x, int gbase, int kk)
{
    const uint64_t *P = Tab1<W>::P();
    p1::Acc160 a = {{0, 0, 0, 0, 0}};
#pragma unroll
    for (int j = 0; j < W; j++) p1::acc160_mul_add(a, shfl_u64(x, gbase + j), __ldg(P + j * W + kk));
    return p1::acc160_reduce(a);
}

// The Poseidon1 permutation (poseidon1.cuh's round structure: add C_0; rounds 0-3 x^7 + next
// constants, M (P after round 3); 22 sparse partial rounds before round 4; rounds 4-7 x^7 +
// constants (none after round 7), M) on the group's state, lane k holding word k.
template <int W>
__device__ __forceinline__ uint64_t permute1(uint64_t x, int gbase, int k)
{
    constexpr int G = Tab<W>::G;
    const bool live = k < W;
    const int kk = live ? k : 0;
    const uint64_t *C = Tab1<W>::C();
    const uint64_t *S = Tab1<W>::S();
    x = live ? gl::add_c(x, __ldg(C + kk)) : 0ull;
#pragma unroll 1
    for (int r = 0; r < 8; r++) {
        if (r == 4) {
#pragma unroll 1
            for (int pr = 0; pr < NPARTIAL; pr++) {
                const uint64_t *Sr = S + (2 * W - 1) * pr;
                const uint64_t x0 = shfl_u64(gl::add_c(gl::pow7(x), __ldg(C + 5 * W + pr)), gbase);
                // x0' = <(x0, x_1..), Sr[0..W)>: one product per lane, summed over the group
                const uint64_t term = live ? gl::mul(k == 0 ? x0 : x, __ldg(Sr + kk)) : 0ull;
                const gl::Acc sum = xor_sum<0, (G == 16 ? 4 : 3)>(gl::acc(term));
                x = k == 0 ? gl::acc_reduce(sum) : (live ? gl::mul_add(x0, __ldg(Sr + W - 1 + kk), x) : 0ull);
            }
        }
        x = gl::pow7(x);
        if (r < 7) x = gl::add_c(x, __ldg(C + (r < 4 ? (r + 1) * W : 5 * W + NPARTIAL + (r - 4) * W) + kk));
        x = r == 3 ? mvp_full1<W>(x, gbase, kk) : mvp_small1<W>(x, gbase, kk);
        if (!live) x = 0;
    }
    return x;
}

template <int W, int FAM>
__device__ __forceinline__ uint64_t permute_fam(uint64_t x, int gbase, int k)
{
    if constexpr (FAM == 1)
        return permute1<W>(x, gbase, k);
    else
        return permute<W>(x, gbase, k);
}

// ---------------------------------------------------------------------------------
// Kernels.  CTAs of CTA_THREADS threads = CTA_THREADS / G states.
// ---------------------------------------------------------------------------------
constexpr int CTA_THREADS = 256;
constexpr int TAIL_THREADS = 1024;

// Parent i of a tree level (semantics of merkle::node_one): the W = 4 * arity child words, zero
// past `pending`; the last parent writes the level's `pad` zero digests after its children.
template <int W, int FAM>
__device__ __forceinline__ void node_group(uint64_t *__restrict__ level, uint64_t pending, uint64_t pad,
                                          uint64_t parents, uint64_t *__restrict__ out, uint64_t i, int gbase, int k)
{
    constexpr uint64_t ARITY = W / 4;
    const bool valid = i < parents;
    uint64_t x = 0;
    if (valid && k < W && i * ARITY + (uint64_t)(k >> 2) < pending) x = level[i * W + k];
    if (valid && i == parents - 1 && (uint64_t)k < pad * 4) level[pending * 4 + k] = 0;
    x = permute_fam<W, FAM>(x, gbase, k);
    if (valid && k < 4) out[i * 4 + k] = gl::canon(x);
}

template <int W, int FAM = 2>
__global__ void __launch_bounds__(CTA_THREADS) node_coop_kernel(uint64_t *__restrict__ level, uint64_t pending,
                                                                uint64_t pad, uint64_t parents,
                                                                uint64_t *__restrict__ out)
{
    constexpr int G = Tab<W>::G;
    const int lane = threadIdx.x & 31;
    const uint64_t i = ((uint64_t)blockIdx.x * CTA_THREADS + threadIdx.x) / G;
    node_group<W, FAM>(level, pending, pad, parents, out, i, lane & ~(G - 1), lane & (G - 1));
}

// Every remaining level of a tree whose current level has `pending` digests at `level`, in one
// CTA (the level loop runs inside; a barrier separates the levels).  Used once a level has at
// most TAIL_THREADS / G parents.
template <int W, int FAM = 2>
__global__ void __launch_bounds__(TAIL_THREADS) tree_tail_kernel(uint64_t *level, uint64_t pending)
{
    constexpr int G = Tab<W>::G;
    constexpr uint64_t ARITY = W / 4;
    const int lane = threadIdx.x & 31;
    const uint64_t i = threadIdx.x / G;
    while (pending > 1) {
        const uint64_t pad = (ARITY - pending % ARITY) % ARITY;
        const uint64_t parents = (pending + ARITY - 1) / ARITY;
        uint64_t *out = level + (pending + pad) * 4;
        node_group<W, FAM>(level, pending, pad, parents, out, i, lane & ~(G - 1), lane & (G - 1));
        __syncthreads();
        level = out;
        pending = parents;
    }
}

// Row sponge of row `row` (semantics of merkle::leaf_row): the capacity starts at zero; each block
// puts the next RATE columns (zero past the last) in lanes [0, RATE) and the previous output words
// 0..3 in the capacity lanes; the digest is words 0..3.
template <int W, int FAM = 2>
__global__ void __launch_bounds__(CTA_THREADS) leaf_coop_kernel(uint64_t *__restrict__ digests,
                                                                const uint64_t *__restrict__ src, uint64_t rs,
                                                                uint64_t cs, uint64_t ncols, uint64_t nrows)
{
    constexpr int G = Tab<W>::G;
    constexpr int RATE = W - 4;
    const int lane = threadIdx.x & 31;
    const int gbase = lane & ~(G - 1), k = lane & (G - 1);
    const uint64_t row = ((uint64_t)blockIdx.x * CTA_THREADS + threadIdx.x) / G;
    const bool valid = row < nrows;
    const uint64_t *p = src + (valid ? row : 0) * rs;
    uint64_t x = 0;
    for (uint64_t done = 0; done < ncols; done += RATE) {
        const uint64_t prev = shfl_u64(x, gbase + (k >= RATE && k < W ? k - RATE : 0));
        if (k < RATE)
            x = (valid && done + k < ncols) ? __ldg(p + (done + k) * cs) : 0ull;
        else if (k < W)
            x = done ? prev : 0ull;
        else
            x = 0;
        x = permute_fam<W, FAM>(x, gbase, k);
    }
    if (valid && k < 4) digests[row * 4 + k] = gl::canon(x);
}

}  // namespace coop
