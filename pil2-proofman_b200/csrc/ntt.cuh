// Low-degree extension of Goldilocks columns on the device.
//
// out[j] = p(7 * w_NExt^j), where p interpolates the column on <w_N> and w_k is the
// reference's W[log2 k] (goldilocks_base_field.cpp:11-44); NTT_Goldilocks::LDE
// (ntt_goldilocks.cpp:369-404) is the CPU statement of the same map.
//
// Data layout: columns are contiguous (column-major, element (row, col) at col*stride + row).
// Plan for one column of N = 2^lg rows and blowup B = 2^b:
//   1. inverse DIF NTT of size N (natural in, bit-reversed out), in windows of <= 12 bits;
//      the last window scales position p by N^-1 * 7^bitrev(p), so position p then holds
//      coefficient c_i * 7^i with i = bitrev(p);
//   2. forward DIT NTT of size N*B (bit-reversed in, natural out).  In bit-reversed order
//      the zero-padded coefficient vector is nonzero only at multiples of B, and its first
//      b butterfly stages just copy, so the first window reads position P from p = P >> b
//      and starts at stage b.  The last window writes canonical values.
// A window covering butterfly stages [s0, s0+k) is a batch of independent 2^k-point
// transforms over elements at stride 2^s0.  One CTA loads a 2^k x L tile (L consecutive
// low-index lanes) into shared memory, applies the single inter-window twiddle
// w_{2^(s0+k)}^(bitrev_k(mid)*lo) per element (before a DIT window, after a DIF window),
// formed from a two-level table of w_{2^26} powers, and runs the k radix-2 stages as
// register radix-16 phases (pass16_kernel below).
#pragma once
#include "gl64.cuh"
#include "prof.cuh"
#include "transpose_tma.cuh"

#include <atomic>
#include <map>
#include <mutex>

#define NTT_KMAX 12   // widest window (phase twiddles are powers of w_4096)
#define NTT_TWLG 26   // inter-window twiddles: powers of w_{2^26}; transforms up to 2^26 points
#define NTT_TILE_MAX 8192

__device__ uint64_t g_ntt_tw_lo_fwd[1 << 13];
__device__ uint64_t g_ntt_tw_hi_fwd[1 << 13];
__device__ uint64_t g_ntt_tw_lo_inv[1 << 13];
__device__ uint64_t g_ntt_tw_hi_inv[1 << 13];
__device__ uint64_t g_ntt_sh_lo_n[(NTT_TWLG + 1) << 12];  // 7^j * 2^-lg at [lg * 4096 + j]
__device__ uint64_t g_ntt_sh_hi[1 << 14];  // 7^(4096 j)

namespace ntt {

enum { POST_NONE = 0, POST_COSET = 1, POST_CANON = 2 };

struct Pass {
    const uint64_t *src;
    uint64_t *dst;
    uint64_t src_cs, dst_cs;  // column strides, elements
    uint32_t lg;              // log2 of the transform length (dst positions)
    uint32_t s0, k, lgL;      // window: stages [s0, s0+k), 2^lgL lanes per tile
    uint32_t rep;             // source position = dst position >> rep
    uint32_t dif;             // 1: inverse DIF window, 0: forward DIT window
    uint32_t post;            // POST_*
    uint32_t gshift;          // source index = ((dst position >> rep) << gshift) + goff
    uint64_t goff;
    uint64_t scale;           // loads multiplied by this factor (0: no scaling)
};

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, uint32_t bits)
{
    return bits ? (__brev(x) >> (32 - bits)) : 0u;
}

__device__ __forceinline__ uint64_t big_twiddle(uint64_t e, bool inv)
{
    const uint64_t *lo = inv ? g_ntt_tw_lo_inv : g_ntt_tw_lo_fwd;
    const uint64_t *hi = inv ? g_ntt_tw_hi_inv : g_ntt_tw_hi_fwd;
    return gl::mul(__ldg(lo + (e & 8191)), __ldg(hi + (e >> 13)));
}

// ---------------------------------------------------------------------------------
// Window kernel with register radix-16 phases.
//
// The 2^k-point transform of a window is split into phases of r <= 4 stages.  In a
// phase each thread takes the 2^r elements of one sub-transform (mid = hi|j<<pb|lo_m),
// applies the phase twiddle w_{2^(pb+r)}^(bitrev_r(j)*lo_m) (before, DIT; after, DIF),
// and runs the r radix-2 stages in registers (roots w_2..w_16 are powers of 2^12: shifts);
// shared memory is touched once per phase instead of once per stage.  Shared memory is
// padded by one word per 16 (index i -> i + i/16) so that a thread's 16 contiguous
// elements of the first phase sit in different banks from its neighbours'.
// ---------------------------------------------------------------------------------

__device__ uint64_t g_ntt_w4096_fwd[4096];  // w_4096^i
__device__ uint64_t g_ntt_w4096_inv[4096];  // w_4096^-i

__device__ __forceinline__ uint32_t pad16(uint32_t i) { return i + (i >> 4); }

// x * w_16^idx = x * 2^(12 idx) (idx constant once the butterfly loops are unrolled)
__device__ __forceinline__ uint64_t mul_root16(uint64_t x, int idx)
{
    switch (idx) {
    case 1: return gl::mul_pow2<12>(x);
    case 2: return gl::mul_pow2<24>(x);
    case 3: return gl::mul_pow2<36>(x);
    case 4: return gl::mul_pow2<48>(x);
    case 5: return gl::mul_pow2<60>(x);
    case 6: return gl::mul_pow2<72>(x);
    case 7: return gl::mul_pow2<84>(x);
    default: return x;
    }
}

// Forward radix-2^R DIT network.  The twiddled operand is made canonical, so the butterfly's add
// and subtract each need one carry fold; the roots w_16^idx = 2^(12 idx) are shift multiplies,
// and those of idx 6 and 7 (2^72, 2^84: a product and a subtraction) are canonical already.
template <int R, bool INV>
__device__ __forceinline__ void radix_dit(uint64_t (&v)[16])
{
    static_assert(!INV, "the DIT network runs forward transforms");
#pragma unroll
    for (int u = 0; u < R; u++) {
        const int h = 1 << u;
#pragma unroll
        for (int j = 0; j < (1 << R); j++) {
            if (j & h) continue;
            const int e = j & (h - 1);
            uint64_t x = v[j + h];
            if (e) x = mul_root16(x, e << (3 - u));
            if ((e << (3 - u)) < 6) x = gl::canon(x);
            const uint64_t y = v[j];
            v[j] = gl::add_c(y, x);
            v[j + h] = gl::sub_c(y, x);
        }
    }
}

// Inverse radix-2^R DIF network.  w_16^-idx = -2^(96 - 12 idx), so a twiddled difference is
// (x - y) * 2^(96 - 12 idx), taken with y canonical; the untwiddled y - x with x canonical.  Either
// way the sum and the difference need one carry fold each.
template <int R, bool INV>
__device__ __forceinline__ void radix_dif(uint64_t (&v)[16])
{
    static_assert(INV, "the DIF network runs inverse transforms");
#pragma unroll
    for (int u = R - 1; u >= 0; u--) {
        const int h = 1 << u;
#pragma unroll
        for (int j = 0; j < (1 << R); j++) {
            if (j & h) continue;
            const int e = j & (h - 1);
            if (e) {
                const uint64_t y = gl::canon(v[j]), x = v[j + h];
                v[j] = gl::add_c(x, y);
                v[j + h] = mul_root16(gl::sub_c(x, y), 8 - (e << (3 - u)));
            } else {
                const uint64_t y = v[j], x = gl::canon(v[j + h]);
                v[j] = gl::add_c(y, x);
                v[j + h] = gl::sub_c(y, x);
            }
        }
    }
}

template <int R, bool DIF>
__device__ __forceinline__ void radix_phase(uint64_t *sm, uint32_t k, uint32_t lgL, uint32_t pb)
{
    constexpr int NR = 1 << R;
    const uint32_t T = 1u << (k + lgL);
    const uint32_t Lm = (1u << lgL) - 1;
    const uint64_t *wtab = DIF ? g_ntt_w4096_inv : g_ntt_w4096_fwd;
    const uint32_t wsh = 12 - pb - R;  // w_{2^(pb+R)} = w_4096^(2^wsh)
    for (uint32_t th = threadIdx.x; th < (T >> R); th += blockDim.x) {
        const uint32_t l = th & Lm, g = th >> lgL;
        const uint32_t lo_m = g & ((1u << pb) - 1), hi_m = g >> pb;
        const uint32_t mbase = (hi_m << (pb + R)) | lo_m;
        uint64_t v[16];
#pragma unroll
        for (int j = 0; j < NR; j++) v[j] = sm[pad16(((mbase | ((uint32_t)j << pb)) << lgL) | l)];
        if (!DIF) {
            if (pb && lo_m) {
#pragma unroll
                for (int j = 1; j < NR; j++) {
                    const uint32_t br = __brev((uint32_t)j) >> (32 - R);
                    v[j] = gl::mul(v[j], __ldg(wtab + (((br * lo_m) << wsh) & 4095)));
                }
            }
            radix_dit<R, false>(v);
        } else {
            radix_dif<R, true>(v);
            if (pb && lo_m) {
#pragma unroll
                for (int j = 1; j < NR; j++) {
                    const uint32_t br = __brev((uint32_t)j) >> (32 - R);
                    v[j] = gl::mul(v[j], __ldg(wtab + (((br * lo_m) << wsh) & 4095)));
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NR; j++) sm[pad16(((mbase | ((uint32_t)j << pb)) << lgL) | l)] = v[j];
    }
}

template <bool DIF>
__device__ __forceinline__ void run_phases(uint64_t *sm, uint32_t k, uint32_t lgL)
{
    // phases of 4 stages from the low mid bits (DIT) or from the high ones (DIF); the odd
    // remainder is the last DIT phase / the first DIF phase
    const uint32_t full = k >> 2, rem = k & 3;
    if (!DIF) {
        for (uint32_t ph = 0; ph < full; ph++) {
            radix_phase<4, false>(sm, k, lgL, 4 * ph);
            __syncthreads();
        }
        const uint32_t pb = 4 * full;
        if (rem == 1) radix_phase<1, false>(sm, k, lgL, pb);
        if (rem == 2) radix_phase<2, false>(sm, k, lgL, pb);
        if (rem == 3) radix_phase<3, false>(sm, k, lgL, pb);
        if (rem) __syncthreads();
    } else {
        const uint32_t pb = 4 * full;
        if (rem == 1) radix_phase<1, true>(sm, k, lgL, pb);
        if (rem == 2) radix_phase<2, true>(sm, k, lgL, pb);
        if (rem == 3) radix_phase<3, true>(sm, k, lgL, pb);
        if (rem) __syncthreads();
        for (int ph = (int)full - 1; ph >= 0; ph--) {
            radix_phase<4, true>(sm, k, lgL, 4 * ph);
            __syncthreads();
        }
    }
}

// One CTA: tile `tile` of column `col` of the window described by `a`.
__device__ __forceinline__ void pass16_body(const Pass &a, uint64_t tile, uint64_t col)
{
    extern __shared__ uint64_t sm[];
    const uint32_t k = a.k, lgL = a.lgL, s0 = a.s0;
    const uint32_t T = 1u << (k + lgL);
    const uint32_t Lm = (1u << lgL) - 1;
    const uint32_t nlob = s0 - lgL;
    const uint64_t hi = tile >> nlob;
    const uint64_t lob = tile & ((1ull << nlob) - 1);
    const uint64_t base = (hi << (s0 + k)) | (lob << lgL);
    const uint64_t *S = a.src + col * a.src_cs;
    uint64_t *D = a.dst + col * a.dst_cs;
    const bool inv = a.dif != 0;
    const uint32_t tw_shift = NTT_TWLG - s0 - k;

    for (uint32_t q = threadIdx.x; q < T; q += blockDim.x) {
        const uint64_t pos = base | ((uint64_t)(q >> lgL) << s0) | (q & Lm);
        uint64_t v = S[((pos >> a.rep) << a.gshift) + a.goff];
        if (a.scale) v = gl::mul(v, a.scale);
        if (!inv && s0 > 0) {
            const uint64_t lo = (lob << lgL) | (q & Lm);
            const uint64_t E = (uint64_t)brev_bits(q >> lgL, k) * lo;
            if (E) v = gl::mul(v, big_twiddle(E << tw_shift, false));
        }
        sm[pad16(q)] = v;
    }
    __syncthreads();
    if (inv)
        run_phases<true>(sm, k, lgL);
    else
        run_phases<false>(sm, k, lgL);
    for (uint32_t q = threadIdx.x; q < T; q += blockDim.x) {
        const uint64_t pos = base | ((uint64_t)(q >> lgL) << s0) | (q & Lm);
        uint64_t v = sm[pad16(q)];
        if (inv && s0 > 0) {
            const uint64_t lo = (lob << lgL) | (q & Lm);
            const uint64_t E = (uint64_t)brev_bits(q >> lgL, k) * lo;
            if (E) v = gl::mul(v, big_twiddle(E << tw_shift, true));
        }
        if (a.post == POST_COSET) {
            const uint32_t br = brev_bits((uint32_t)pos, a.lg);
            const uint64_t f =
                gl::mul(__ldg(g_ntt_sh_lo_n + (a.lg << 12) + (br & 4095)), __ldg(g_ntt_sh_hi + (br >> 12)));
            v = gl::mul(v, f);
        } else if (a.post == POST_CANON) {
            v = gl::canon(v);
        }
        D[pos] = v;
    }
}

// two CTAs of 512 threads per SM (<= 64 registers): one CTA's global loads overlap the other's
// shared-memory phases
__global__ void __launch_bounds__(512, 2) pass16_kernel(Pass a) { pass16_body(a, blockIdx.x, blockIdx.y); }

// ---------------------------------------------------------------------------------
// Fixed-shape window kernels.  The same computation as pass16_body with the window's
// width K and lane count 2^LGL known at compile time: every loop has a constant trip
// count, every phase's shared-memory addresses are one per-thread base plus constant
// offsets, and positions are 32-bit (transforms are at most 2^26 points).  The generic
// kernel above serves the shapes that are not instantiated.
// ---------------------------------------------------------------------------------

template <int K, int LGL>
struct Shape {
    static constexpr int T = 1 << (K + LGL);
    static constexpr int NT = (T / 16) < 32 ? 32 : (T / 16) > 512 ? 512 : (T / 16);
};

// padded shared-memory index of element (base + j * 2^M) for base with zero bits in
// [M, M + R): for M >= 4 the padding of the sum splits, (b + j*2^M) + (b + j*2^M)/16 =
// pad16(b) + j*(2^M + 2^(M-4)), so offsets are compile-time constants.
template <int M>
__device__ __forceinline__ uint32_t pad_off(uint32_t pbase, uint32_t base, int j)
{
    if (M >= 4) return pbase + (uint32_t)j * ((1u << M) + (1u << (M >= 4 ? M - 4 : 0)));
    return pad16(base + ((uint32_t)j << M));
}

template <int R, bool DIF, int K, int LGL, int PB>
__device__ __forceinline__ void radix_phase_fixed(uint64_t *sm)
{
    constexpr int NR = 1 << R;
    constexpr int G = Shape<K, LGL>::T >> R;  // sub-transforms in the tile
    constexpr int NT = Shape<K, LGL>::NT;
    constexpr int IT = (G + NT - 1) / NT;
    constexpr int M = PB + LGL;
    const uint64_t *wtab = DIF ? g_ntt_w4096_inv : g_ntt_w4096_fwd;
    constexpr int WSH = 12 - PB - R;  // w_{2^(PB+R)} = w_4096^(2^WSH)
#pragma unroll
    for (int it = 0; it < IT; it++) {
        const uint32_t th = threadIdx.x + (uint32_t)it * NT;
        if ((G % NT) != 0 && th >= (uint32_t)G) break;
        const uint32_t l = th & ((1u << LGL) - 1), g = th >> LGL;
        const uint32_t lo_m = g & ((1u << PB) - 1), hi_m = g >> PB;
        const uint32_t base = (((hi_m << (PB + R)) | lo_m) << LGL) | l;
        const uint32_t pbase = pad16(base);
        uint64_t v[16];
#pragma unroll
        for (int j = 0; j < NR; j++) v[j] = sm[pad_off<M>(pbase, base, j)];
        if (!DIF) {
            if (PB && lo_m) {
#pragma unroll
                for (int j = 1; j < NR; j++) {
                    const uint32_t br = __brev((uint32_t)j) >> (32 - R);
                    v[j] = gl::mul(v[j], __ldg(wtab + (((br * lo_m) << WSH) & 4095)));
                }
            }
            radix_dit<R, false>(v);
        } else {
            radix_dif<R, true>(v);
            if (PB && lo_m) {
#pragma unroll
                for (int j = 1; j < NR; j++) {
                    const uint32_t br = __brev((uint32_t)j) >> (32 - R);
                    v[j] = gl::mul(v[j], __ldg(wtab + (((br * lo_m) << WSH) & 4095)));
                }
            }
        }
#pragma unroll
        for (int j = 0; j < NR; j++) sm[pad_off<M>(pbase, base, j)] = v[j];
    }
}

// Radix of the fixed kernels' phases: 2^NTT_PHASE_BITS points per thread and phase.
constexpr int NTT_PHASE_BITS = 4;

// DIT: full phases from the low mid bits, then the remainder; DIF: the reverse order
template <bool DIF, int K, int LGL, int PH>
__device__ __forceinline__ void phases_fixed(uint64_t *sm)
{
    constexpr int RP = NTT_PHASE_BITS;
    constexpr int FULL = K / RP, REM = K % RP;
    if constexpr (!DIF) {
        if constexpr (PH < FULL) {
            radix_phase_fixed<RP, false, K, LGL, RP * PH>(sm);
            __syncthreads();
            phases_fixed<false, K, LGL, PH + 1>(sm);
        } else if constexpr (REM != 0) {
            radix_phase_fixed<REM, false, K, LGL, RP * FULL>(sm);
            __syncthreads();
        }
    } else {
        // PH counts down from FULL (the remainder phase) to 0
        if constexpr (PH == FULL) {
            if constexpr (REM != 0) {
                radix_phase_fixed<REM, true, K, LGL, RP * FULL>(sm);
                __syncthreads();
            }
            if constexpr (FULL > 0) phases_fixed<true, K, LGL, FULL - 1>(sm);
        } else {
            radix_phase_fixed<RP, true, K, LGL, RP * PH>(sm);
            __syncthreads();
            if constexpr (PH > 0) phases_fixed<true, K, LGL, PH - 1>(sm);
        }
    }
}

__host__ __device__ constexpr int log2_const(int x) { return x <= 1 ? 0 : 1 + log2_const(x >> 1); }

// Thread / iteration decomposition of a fixed-shape tile.  Element q = threadIdx.x + it * NT of the
// tile is (mid, lane) = (q >> LGL, q & Lm).  When NT is a multiple of 2^LGL (SPLIT) a thread keeps
// one lane, and mid = M0 + it * 2^MB with M0 = threadIdx.x >> LGL below 2^MB: the low MB bits of
// mid come from the thread, the high LOG_IT bits from the iteration, so
//   brev_K(mid) = (brev_MB(M0) << LOG_IT) + brev_LOG_IT(it).
// Any factor w^(brev_K(mid) * c) is then a per-thread constant times a power of w^c whose exponent
// is brev_LOG_IT(it): visiting the iterations in bit-reversed order makes that exponent count up,
// and the factors are running products (no table lookups in the loop).
template <int K, int LGL>
struct Iter {
    static constexpr int T = Shape<K, LGL>::T, NT = Shape<K, LGL>::NT, IT = (T + NT - 1) / NT;
    static constexpr int LOG_NT = log2_const(NT);
    static constexpr bool SPLIT = (T % NT == 0) && LOG_NT >= LGL && (1 << (K + LGL)) == T;
    static constexpr int MB = SPLIT ? LOG_NT - LGL : 0;
    static constexpr int LOG_IT = SPLIT ? K - MB : 0;
    static constexpr int CH = IT < 4 ? IT : 4;  // independent product chains of the load side (latency)
    // the store side holds its chains while the tile is read back: two keep the inverse windows
    // inside the 64-register budget
    static constexpr int CH_STORE = IT < 2 ? IT : 2;
};

// Running powers f(it') = A * B^it' for it' = 0 .. IT-1, as CH interleaved chains: chain c yields
// it' = c, c + CH, c + 2 CH, ...  next(c) returns chain c's current value and advances it.
template <int CH>
struct Powers {
    uint64_t v[CH];
    uint64_t step;  // B^CH
    __device__ __forceinline__ void init(uint64_t A, uint64_t B)
    {
        v[0] = A;
#pragma unroll
        for (int c = 1; c < CH; c++) v[c] = gl::mul(v[c - 1], B);
        uint64_t s = B;
#pragma unroll
        for (int c = 1; c < CH; c++) s = gl::mul(s, B);  // B^CH (CH <= 4)
        step = s;
    }
    __device__ __forceinline__ uint64_t next(int c)
    {
        const uint64_t r = v[c];
        v[c] = gl::mul(v[c], step);
        return r;
    }
};

// The inter-window twiddles of this thread's elements, w_{2^(s0+K)}^(brev_K(mid) * lo) (SPLIT shapes).
template <int K, int LGL, int CH>
__device__ __forceinline__ void window_twiddles(Powers<CH> &pw, uint32_t lob, uint32_t tw_shift, bool inv)
{
    using I = Iter<K, LGL>;
    constexpr uint32_t Lm = (1u << LGL) - 1;
    const uint32_t lo = (lob << LGL) | (threadIdx.x & Lm);
    const uint32_t M0 = threadIdx.x >> LGL;
    const uint32_t e0 = (brev_bits(M0, I::MB) << I::LOG_IT) * lo;  // < 2^(s0 + K) <= 2^26
    pw.init(big_twiddle((uint64_t)e0 << tw_shift, inv), big_twiddle((uint64_t)lo << tw_shift, inv));
}

// First forward window of an LDE at blowup 2^LGL (s0 = rep = LGL): the tile's 2^LGL lanes of a mid
// are copies of one source element (the zero padding folded away), lane l twiddled by t^l with
// t = w_{2^(s0+K)}^brev_K(mid).  Each thread loads its sources once (mid = threadIdx.x + i * NT,
// coalesced), forms t as a running product over i in bit-reversed order, and writes all lanes.
template <int K, int LGL>
__device__ __forceinline__ void load_tile_copies(uint64_t *sm, const uint64_t *S, uint32_t base, uint32_t tw_shift)
{
    constexpr int NT = Shape<K, LGL>::NT, LOG_NT = log2_const(NT);
    constexpr int NI = (1 << K) / NT, LOG_NI = K - LOG_NT;  // sources per thread
    constexpr int CH = NI < 4 ? NI : 4;
    static_assert((1 << K) % NT == 0 && K >= LOG_NT, "copy-lane load needs NT | 2^K");
    const uint64_t *src = S + (base >> LGL);
    Powers<CH> pw;
    pw.init(big_twiddle((uint64_t)(brev_bits(threadIdx.x, LOG_NT) << LOG_NI) << tw_shift, false),
            big_twiddle((uint64_t)1 << tw_shift, false));
#pragma unroll 1
    for (int jj = 0; jj < NI; jj += CH) {
#pragma unroll
        for (int c = 0; c < CH; c++) {
            const uint32_t mid = threadIdx.x + brev_bits((uint32_t)(jj + c), LOG_NI) * NT;
            const uint64_t v = src[mid];
            const uint64_t t = pw.next(c);
            uint64_t u = v;
            sm[pad16(mid << LGL)] = v;
#pragma unroll
            for (int l = 1; l < (1 << LGL); l++) {
                u = gl::mul(u, t);
                sm[pad16((mid << LGL) | l)] = u;
            }
        }
    }
}

// Register-path tile load of a fixed-shape window: the gather (with the Q stage's source remap
// and scale), the forward windows' inter-window twiddle, the store to shared memory.  With a SPLIT
// shape the twiddles are running products (Iter); otherwise each is a product of two table entries.
template <int K, int LGL, bool DIF>
__device__ __forceinline__ void load_tile(uint64_t *sm, const Pass &a, const uint64_t *S, uint32_t base,
                                          uint32_t lob, uint32_t s0, uint32_t tw_shift)
{
    using I = Iter<K, LGL>;
    constexpr int T = I::T, NT = I::NT, IT = I::IT;
    constexpr uint32_t Lm = (1u << LGL) - 1;
    const uint32_t rep = a.rep, gshift = a.gshift, goff = (uint32_t)a.goff;
    const bool tw = !DIF && s0 > 0;
    if constexpr (!DIF && LGL >= 1 && LGL <= 2 && K >= log2_const(Shape<K, LGL>::NT)) {
        if (rep == LGL && s0 == LGL && gshift == 0 && goff == 0 && a.scale == 0) {
            load_tile_copies<K, LGL>(sm, S, base, tw_shift);
            return;
        }
    }
    if constexpr (I::SPLIT) {
        Powers<I::CH> pw;
        if (tw) window_twiddles<K, LGL, I::CH>(pw, lob, tw_shift, false);
#pragma unroll 1
        for (int jj = 0; jj < IT; jj += I::CH) {
#pragma unroll
            for (int c = 0; c < I::CH; c++) {
                const uint32_t it = brev_bits((uint32_t)(jj + c), I::LOG_IT);
                const uint32_t q = threadIdx.x + it * NT;
                const uint32_t pos = base | ((q >> LGL) << s0) | (q & Lm);
                uint64_t v = S[((pos >> rep) << gshift) + goff];
                if (a.scale) v = gl::mul(v, a.scale);
                if (tw) v = gl::mul(v, pw.next(c));
                sm[pad16(q)] = v;
            }
        }
    } else {
#pragma unroll 4  // full unrolling hoists all 16 loads of a thread and spills at 64 registers
        for (int it = 0; it < IT; it++) {
            const uint32_t q = threadIdx.x + (uint32_t)it * NT;
            if ((T % NT) != 0 && q >= (uint32_t)T) break;
            const uint32_t pos = base | ((q >> LGL) << s0) | (q & Lm);
            uint64_t v = S[((pos >> rep) << gshift) + goff];
            if (a.scale) v = gl::mul(v, a.scale);
            if (tw) {
                const uint32_t lo = (lob << LGL) | (q & Lm);
                const uint32_t E = (__brev(q >> LGL) >> (32 - K)) * lo;
                if (E) v = gl::mul(v, big_twiddle((uint64_t)(E << tw_shift), false));
            }
            sm[pad16(q)] = v;
        }
    }
}

// Tile store of a fixed-shape window: the inverse windows' inter-window twiddle or, in the last
// inverse window (s0 = 0, LGL = 0), the coset scale 7^bitrev(pos) / N; canonical values after the
// last forward window.
template <int K, int LGL, bool DIF>
__device__ __forceinline__ void store_tile(const uint64_t *sm, const Pass &a, uint64_t *D, uint32_t base, uint32_t lob,
                                           uint32_t s0, uint32_t tw_shift)
{
    using I = Iter<K, LGL>;
    constexpr int T = I::T, NT = I::NT, IT = I::IT;
    constexpr uint32_t Lm = (1u << LGL) - 1;
    const bool tw = DIF && s0 > 0;
    const uint32_t post = a.post;
    if constexpr (I::SPLIT) {
        Powers<I::CH_STORE> pw;
        if (tw) {
            window_twiddles<K, LGL, I::CH_STORE>(pw, lob, tw_shift, true);
        } else if (post == POST_COSET) {
            // pos = base | q (s0 = 0, LGL = 0), base = hi << K: brev_lg(pos) = brev_lg(base) +
            // ((brev_MB(tid) << LOG_IT) + brev_LOG_IT(it)) << (lg - K)
            const uint32_t lg = a.lg, up = lg - K;
            const uint32_t e0 = brev_bits(base, lg) + ((brev_bits(threadIdx.x, I::MB) << I::LOG_IT) << up);
            const uint64_t c0 =
                gl::mul(__ldg(g_ntt_sh_lo_n + (lg << 12) + (e0 & 4095)), __ldg(g_ntt_sh_hi + (e0 >> 12)));
            const uint32_t es = 1u << up;  // 7^(2^up), without the 1/N of the lg table (lg 0: 2^0)
            const uint64_t st = gl::mul(__ldg(g_ntt_sh_lo_n + (es & 4095)), __ldg(g_ntt_sh_hi + (es >> 12)));
            pw.init(c0, st);
        }
#pragma unroll 1
        for (int jj = 0; jj < IT; jj += I::CH_STORE) {
#pragma unroll
            for (int c = 0; c < I::CH_STORE; c++) {
                const uint32_t it = brev_bits((uint32_t)(jj + c), I::LOG_IT);
                const uint32_t q = threadIdx.x + it * NT;
                const uint32_t pos = base | ((q >> LGL) << s0) | (q & Lm);
                uint64_t v = sm[pad16(q)];
                if (tw || post == POST_COSET)
                    v = gl::mul(v, pw.next(c));
                else if (post == POST_CANON)
                    v = gl::canon(v);
                D[pos] = v;
            }
        }
    } else {
#pragma unroll 4  // full unrolling hoists all 16 loads of a thread and spills at 64 registers
        for (int it = 0; it < IT; it++) {
            const uint32_t q = threadIdx.x + (uint32_t)it * NT;
            if ((T % NT) != 0 && q >= (uint32_t)T) break;
            const uint32_t pos = base | ((q >> LGL) << s0) | (q & Lm);
            uint64_t v = sm[pad16(q)];
            if (tw) {
                const uint32_t lo = (lob << LGL) | (q & Lm);
                const uint32_t E = (__brev(q >> LGL) >> (32 - K)) * lo;
                if (E) v = gl::mul(v, big_twiddle((uint64_t)(E << tw_shift), true));
            }
            if (post == POST_COSET) {
                const uint32_t br = brev_bits(pos, a.lg);
                const uint64_t f =
                    gl::mul(__ldg(g_ntt_sh_lo_n + (a.lg << 12) + (br & 4095)), __ldg(g_ntt_sh_hi + (br >> 12)));
                v = gl::mul(v, f);
            } else if (post == POST_CANON) {
                v = gl::canon(v);
            }
            D[pos] = v;
        }
    }
}

// One CTA of Shape<K,LGL>::NT threads: tile `tile` of column `col` of the window `a`, whose
// direction (a.dif) is DIF.  The direction is a template parameter so that each instantiation
// holds only its own load path and twiddle placement.
template <int K, int LGL, bool DIF>
__device__ __forceinline__ void pass_fixed_body(const Pass &a, uint32_t tile, uint64_t col)
{
    extern __shared__ uint64_t sm[];
    constexpr int T = Shape<K, LGL>::T, NT = Shape<K, LGL>::NT;
    constexpr int IT = (T + NT - 1) / NT;
    constexpr uint32_t Lm = (1u << LGL) - 1;
    const uint32_t s0 = a.s0;
    const uint32_t nlob = s0 - LGL;
    const uint32_t hi = tile >> nlob, lob = tile & ((1u << nlob) - 1);
    const uint32_t base = (hi << (s0 + K)) | (lob << LGL);
    const uint64_t *S = a.src + col * a.src_cs;
    uint64_t *D = a.dst + col * a.dst_cs;
    constexpr bool inv = DIF;
    const uint32_t tw_shift = NTT_TWLG - s0 - K;
    const uint32_t rep = a.rep, gshift = a.gshift, goff = (uint32_t)a.goff;

    if (inv && rep == 0 && gshift == 0 && goff == 0 && a.scale == 0) {
        // Inverse (DIF) windows load a plain gather: every element of the tile goes straight to
        // shared memory with cp.async (no registers, all of a thread's copies in flight at once).
        // The forward windows keep the register path: their load-time twiddle as a separate
        // shared-memory pass measured slower.
#pragma unroll
        for (int it = 0; it < IT; it++) {
            const uint32_t q = threadIdx.x + (uint32_t)it * NT;
            if ((T % NT) != 0 && q >= (uint32_t)T) break;
            const uint32_t pos = base | ((q >> LGL) << s0) | (q & Lm);
            const uint32_t dst = (uint32_t)__cvta_generic_to_shared(sm + pad16(q));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(S + pos) : "memory");
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    } else {
        load_tile<K, LGL, DIF>(sm, a, S, base, lob, s0, tw_shift);
    }
    __syncthreads();
    if constexpr (inv)
        phases_fixed<true, K, LGL, K / NTT_PHASE_BITS>(sm);
    else
        phases_fixed<false, K, LGL, 0>(sm);
    store_tile<K, LGL, DIF>(sm, a, D, base, lob, s0, tw_shift);
}

template <int K, int LGL, bool DIF>
__global__ void __launch_bounds__(Shape<K, LGL>::NT, 1024 / Shape<K, LGL>::NT) pass_fixed_kernel(Pass a)
{
    pass_fixed_body<K, LGL, DIF>(a, blockIdx.x, blockIdx.y);
}

typedef void (*PassKernel)(Pass);

// Instantiated shapes, each in both directions: full 8192-element tiles (K + LGL = 13: every
// window of a large transform but the inverse's first) and single-lane windows (LGL = 0: the
// inverse's first).
template <int K>
inline PassKernel fixed_kernel_k(uint32_t lgL, uint32_t dif)
{
    if (lgL == 13 - K) return dif ? pass_fixed_kernel<K, 13 - K, true> : pass_fixed_kernel<K, 13 - K, false>;
    if (lgL == 0) return dif ? pass_fixed_kernel<K, 0, true> : pass_fixed_kernel<K, 0, false>;
    return nullptr;
}

inline PassKernel fixed_kernel(uint32_t k, uint32_t lgL, uint32_t dif)
{
    switch (k) {
    case 1: return fixed_kernel_k<1>(lgL, dif);
    case 2: return fixed_kernel_k<2>(lgL, dif);
    case 3: return fixed_kernel_k<3>(lgL, dif);
    case 4: return fixed_kernel_k<4>(lgL, dif);
    case 5: return fixed_kernel_k<5>(lgL, dif);
    case 6: return fixed_kernel_k<6>(lgL, dif);
    case 7: return fixed_kernel_k<7>(lgL, dif);
    case 8: return fixed_kernel_k<8>(lgL, dif);
    case 9: return fixed_kernel_k<9>(lgL, dif);
    case 10: return fixed_kernel_k<10>(lgL, dif);
    case 11: return fixed_kernel_k<11>(lgL, dif);
    case 12: return fixed_kernel_k<12>(lgL, dif);
    default: return nullptr;
    }
}

// dynamic shared memory limit of every instantiated shape (tiles above 48 KB need the opt-in)
inline cudaError_t set_fixed_attrs()
{
    for (uint32_t k = 1; k <= NTT_KMAX; k++) {
        const uint32_t shapes[2] = {13 - k, 0};
        for (uint32_t lgL : shapes)
            for (uint32_t dif = 0; dif < 2; dif++) {
                PassKernel kf = fixed_kernel(k, lgL, dif);
                if (!kf) continue;
                const uint32_t T = 1u << (k + lgL);
                cudaError_t e =
                    cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (T + T / 16) * 8);
                if (e != cudaSuccess) return e;
            }
    }
    return cudaSuccess;
}

// row-major (nrows x ncols) -> column-major with column stride dst_cs; one 32x32 tile per
// CTA of 32x8 threads
__device__ __forceinline__ void transpose_tile(uint64_t *__restrict__ dst, const uint64_t *__restrict__ src,
                                               uint64_t nrows, uint64_t ncols, uint64_t dst_cs, uint64_t rtile,
                                               uint64_t ctile)
{
    __shared__ uint64_t tile[32][33];
    const uint64_t r0 = rtile * 32, c0 = ctile * 32;
    const uint32_t tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint64_t r = r0 + ty + 8 * j, c = c0 + tx;
        if (r < nrows && c < ncols) tile[ty + 8 * j][tx] = src[r * ncols + c];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint64_t c = c0 + ty + 8 * j, r = r0 + tx;
        if (r < nrows && c < ncols) dst[c * dst_cs + r] = tile[tx][ty + 8 * j];
    }
}

__global__ void __launch_bounds__(256) transpose_kernel(uint64_t *__restrict__ dst, const uint64_t *__restrict__ src,
                                                        uint64_t nrows, uint64_t ncols, uint64_t dst_cs)
{
    transpose_tile(dst, src, nrows, ncols, dst_cs, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------------ host side ----

// 1 (default): row-major -> column-major transposes stage their tiles with the TMA
// (transpose_tma_kernel) where the shape and alignment allow it; 0: shared-memory tiles loaded by
// the threads (transpose_kernel).  Same values either way.
inline std::atomic<int> &transpose_tma_enabled()
{
    static std::atomic<int> on{1};
    return on;
}

// row-major nrows x ncols -> column-major with column stride dst_cs (one launch)
inline cudaError_t transpose(uint64_t *dst, const uint64_t *src, uint64_t nrows, uint64_t ncols, uint64_t dst_cs,
                             cudaStream_t stream)
{
    if (nrows == 0 || ncols == 0) return cudaSuccess;
    const dim3 grid((unsigned)((nrows + 31) / 32), (unsigned)((ncols + 31) / 32));
    CUtensorMap map;
    if (transpose_tma_enabled().load() && tma_source_map(&map, src, nrows, ncols))
        transpose_tma_kernel<<<grid, dim3(32, 8), 0, stream>>>(dst, map, nrows, ncols, dst_cs);
    else
        transpose_kernel<<<grid, dim3(32, 8), 0, stream>>>(dst, src, nrows, ncols, dst_cs);
    prof::count();
    return cudaGetLastError();
}

struct Window {
    uint32_t s0, k, lgL;
};

// Plan parameters per shape, filled by the autotuner (b200_autotune_lde): the largest first
// window and the largest later windows.  Shapes never tuned use the defaults.
struct Tune {
    uint32_t kfirst = NTT_KMAX, krest = 11;
};

inline std::mutex &tune_mu()
{
    static std::mutex m;
    return m;
}

inline std::map<uint64_t, Tune> &tune_table()
{
    static std::map<uint64_t, Tune> t;
    return t;
}

// column counts are bucketed: the plan depends on the transform length, the grid on the width
inline uint64_t tune_key(uint32_t nBits, uint32_t nBitsExt, uint64_t ncols)
{
    const uint64_t bucket = ncols <= 32 ? 0 : ncols <= 128 ? 1 : ncols <= 512 ? 2 : 3;
    return (uint64_t)nBits | ((uint64_t)nBitsExt << 8) | (bucket << 16);
}

inline Tune tuned(uint32_t nBits, uint32_t nBitsExt, uint64_t ncols)
{
    std::lock_guard<std::mutex> lk(tune_mu());
    auto it = tune_table().find(tune_key(nBits, nBitsExt, ncols));
    return it == tune_table().end() ? Tune{} : it->second;
}

inline void set_tuned(uint32_t nBits, uint32_t nBitsExt, uint64_t ncols, Tune t)
{
    std::lock_guard<std::mutex> lk(tune_mu());
    tune_table()[tune_key(nBits, nBitsExt, ncols)] = t;
}

// Windows covering stages [lo, hi).  The window that starts at `lo` keeps every lower lane
// (lgL = lo) so its tile is one contiguous run; the others take as many lanes as fill an
// 8192-element tile (at most all 2^s0 of them).  kfirst / krest cap the first window and the
// others (the autotuned plan parameters).
inline int plan_windows(uint32_t lo, uint32_t hi, Window *w, int maxw, uint32_t kfirst = NTT_KMAX,
                        uint32_t krest = 11)
{
    int n = 0;
    uint32_t total = hi - lo;
    uint32_t k0 = total;
    if (k0 > kfirst) k0 = kfirst;
    if (k0 > NTT_KMAX) k0 = NTT_KMAX;
    if (k0 + lo > 13) k0 = (lo >= 13) ? 0 : 13 - lo;
    if (k0 == 0 && total > 0) return -1;  // stage offset too large for one tile
    if (krest < 1 || krest > NTT_KMAX) krest = 11;
    w[n++] = Window{lo, k0, lo};
    uint32_t rest = total - k0, s = lo + k0;
    uint32_t np = (rest + krest - 1) / krest;
    for (uint32_t i = 0; i < np; i++) {
        uint32_t k = rest / (np - i) + ((rest % (np - i)) ? 1 : 0);
        uint32_t lgL = 13 - k;  // 2^k x L = 8192-element tiles: L-word contiguous runs
        if (lgL > s) lgL = s;
        if (n >= maxw) return -1;
        w[n++] = Window{s, k, lgL};
        s += k;
        rest -= k;
    }
    return n;
}

inline cudaError_t launch_pass(const Pass &p, uint64_t ncols, cudaStream_t stream)
{
    const uint32_t T = 1u << (p.k + p.lgL);
    const uint64_t tiles = (1ull << p.lg) >> (p.k + p.lgL);
    uint32_t threads = T / 16;  // one radix-16 group per thread and phase
    if (threads < 32) threads = 32;
    if (threads > 512) threads = 512;
    dim3 grid((unsigned)tiles, (unsigned)ncols);
    const size_t smem = (size_t)(T + T / 16) * 8;
    if (PassKernel kf = fixed_kernel(p.k, p.lgL, p.dif)) {
        kf<<<grid, threads, smem, stream>>>(p);
    } else {
        pass16_kernel<<<grid, threads, smem, stream>>>(p);
    }
    prof::count();
    return cudaGetLastError();
}

// Scratch needed by lde(): one column-major copy of the trace.
inline uint64_t lde_scratch_words(uint32_t nBits, uint64_t ncols) { return (1ull << nBits) * ncols; }

// d_lde: column-major NExt x ncols (stride NExt).  d_trace: row-major (trace_rowmajor) or
// column-major with stride N.  d_scratch: lde_scratch_words() words, distinct from d_lde.  For
// column-major input d_scratch may be d_trace itself: every inverse window reads a whole tile
// before writing it back, so the transform then runs in place and leaves the coefficients there;
// with d_scratch distinct the input is left unchanged.  Row-major input is transposed into
// d_scratch first, so there d_scratch must not overlap d_trace.
inline cudaError_t lde(uint64_t *d_lde, const uint64_t *d_trace, bool trace_rowmajor, uint32_t nBits,
                       uint32_t nBitsExt, uint64_t ncols, uint64_t *d_scratch, cudaStream_t stream)
{
    if (ncols == 0) return cudaSuccess;
    if (nBitsExt < nBits || nBitsExt > NTT_TWLG || ncols > 65535) return cudaErrorInvalidValue;
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    const uint32_t b = nBitsExt - nBits;
    cudaError_t err;

    const uint64_t *cur = d_trace;
    uint64_t cur_cs = N;
    if (trace_rowmajor) {
        prof::Scope ps(prof::TRANSPOSE, stream);
        if ((err = transpose(d_scratch, d_trace, N, ncols, N, stream)) != cudaSuccess) return err;
        cur = d_scratch;
    }

    // inverse DIF over [0, nBits), windows applied from the top stage down
    Window w[8];
    const Tune tn = tuned(nBits, nBitsExt, ncols);
    int nw = nBits ? plan_windows(0, nBits, w, 8, tn.kfirst, tn.krest) : 0;
    if (nw < 0) return cudaErrorInvalidValue;
    {
    prof::Scope ps(prof::NTT_INV, stream);
    for (int i = nw - 1; i >= 0; i--) {
        Pass p{};
        p.src = cur;
        p.dst = d_scratch;
        p.src_cs = cur_cs;
        p.dst_cs = N;
        p.lg = nBits;
        p.s0 = w[i].s0;
        p.k = w[i].k;
        p.lgL = w[i].lgL;
        p.rep = 0;
        p.dif = 1;
        p.post = (i == 0) ? POST_COSET : POST_NONE;
        if ((err = launch_pass(p, ncols, stream)) != cudaSuccess) return err;
        cur = d_scratch;
        cur_cs = N;
    }
    }

    // forward DIT over [b, nBitsExt) with replication by 2^b on the first window
    nw = plan_windows(b, nBitsExt, w, 8, tn.kfirst, tn.krest);
    if (nw < 0) return cudaErrorInvalidValue;
    prof::Scope ps(prof::NTT_FWD, stream);
    for (int i = 0; i < nw; i++) {
        Pass p{};
        p.src = (i == 0) ? cur : d_lde;
        p.dst = d_lde;
        p.src_cs = (i == 0) ? cur_cs : NExt;
        p.dst_cs = NExt;
        p.lg = nBitsExt;
        p.s0 = w[i].s0;
        p.k = w[i].k;
        p.lgL = w[i].lgL;
        p.rep = (i == 0) ? b : 0;
        p.dif = 0;
        p.post = (i == nw - 1) ? POST_CANON : POST_NONE;
        if ((err = launch_pass(p, ncols, stream)) != cudaSuccess) return err;
    }
    return cudaSuccess;
}

// Q-stage extension (Starks::computeQ, starks.hpp:186-239; GPU computeQColMajor,
// ntt_goldilocks.cu:1515-1544): q holds qDim columns of NExt evaluations; their inverse NTT
// over NExt gives coefficients c, which are cut into qDeg chunks of N, chunk p scaled by
// S[p] = (7^-1)^(N*p), zero-padded to NExt and forward-transformed; cmQ column p*qDim + k is
// chunk p of limb k.  Here the inverse DIF leaves c in bit-reversed order (position P holds
// NExt*c[bitrev(P)]); the coefficient p*N + i sits at P = (bitrev_n(i) << b) | bitrev_b(p), so the
// first forward window of chunk p gathers positions (q << b) | bitrev_b(p) and scales them by
// S[p]/NExt — the zero padding and the first b forward stages fold away as in lde().
// d_cmq: column-major NExt x (qDeg*qDim); d_q: column-major NExt x qDim (or row-major);
// d_scratch: NExt * qDim words.  Requires qDeg <= NExt/N.
inline cudaError_t lde_q(uint64_t *d_cmq, const uint64_t *d_q, bool q_rowmajor, uint32_t nBits, uint32_t nBitsExt,
                         uint32_t qDeg, uint32_t qDim, uint64_t *d_scratch, cudaStream_t stream)
{
    if (qDim == 0 || qDeg == 0) return cudaSuccess;
    const uint32_t b = nBitsExt - nBits;
    if (nBitsExt < nBits || nBitsExt > NTT_TWLG || (uint64_t)qDeg > (1ull << b)) return cudaErrorInvalidValue;
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    cudaError_t err;
    if (q_rowmajor) {
        prof::Scope ps(prof::TRANSPOSE, stream);
        if ((err = transpose(d_scratch, d_q, NExt, qDim, NExt, stream)) != cudaSuccess) return err;
    } else {
        err = cudaMemcpyAsync(d_scratch, d_q, NExt * qDim * 8, cudaMemcpyDeviceToDevice, stream);
        if (err != cudaSuccess) return err;
    }
    if ((err = cudaGetLastError()) != cudaSuccess) return err;
    Window w[8];
    const Tune tn = tuned(nBitsExt, nBitsExt, qDim);
    int nw = plan_windows(0, nBitsExt, w, 8, tn.kfirst, tn.krest);
    if (nw < 0) return cudaErrorInvalidValue;
    {
        prof::Scope ps(prof::NTT_INV, stream);
        for (int i = nw - 1; i >= 0; i--) {
            Pass p{};
            p.src = d_scratch;
            p.dst = d_scratch;
            p.src_cs = p.dst_cs = NExt;
            p.lg = nBitsExt;
            p.s0 = w[i].s0;
            p.k = w[i].k;
            p.lgL = w[i].lgL;
            p.dif = 1;
            p.post = POST_NONE;
            if ((err = launch_pass(p, qDim, stream)) != cudaSuccess) return err;
        }
    }
    nw = plan_windows(b, nBitsExt, w, 8, tn.kfirst, tn.krest);
    if (nw < 0) return cudaErrorInvalidValue;
    prof::Scope ps(prof::NTT_FWD, stream);
    const uint64_t shift_in = glh::pow(glh::inv(7), N), next_inv = glh::inv(NExt % GL_P);
    uint64_t S = 1;
    for (uint32_t pc = 0; pc < qDeg; pc++) {
        Pass p{};
        p.src = d_scratch;
        p.dst = d_cmq + (uint64_t)pc * qDim * NExt;
        p.src_cs = p.dst_cs = NExt;
        p.lg = nBitsExt;
        p.s0 = w[0].s0;
        p.k = w[0].k;
        p.lgL = w[0].lgL;
        p.rep = b;
        p.gshift = b;
        uint64_t br = 0;
        for (uint32_t t = 0; t < b; t++) br |= (uint64_t)((pc >> t) & 1) << (b - 1 - t);
        p.goff = br;
        p.scale = glh::mul(S, next_inv);  // nonzero: a product of nonzero field elements
        p.post = (nw == 1) ? POST_CANON : POST_NONE;
        if ((err = launch_pass(p, qDim, stream)) != cudaSuccess) return err;
        S = glh::mul(S, shift_in);
    }
    for (int i = 1; i < nw; i++) {
        Pass p{};
        p.src = d_cmq;
        p.dst = d_cmq;
        p.src_cs = p.dst_cs = NExt;
        p.lg = nBitsExt;
        p.s0 = w[i].s0;
        p.k = w[i].k;
        p.lgL = w[i].lgL;
        p.post = (i == nw - 1) ? POST_CANON : POST_NONE;
        if ((err = launch_pass(p, (uint64_t)qDeg * qDim, stream)) != cudaSuccess) return err;
    }
    return cudaSuccess;
}

// Twiddle and coset tables, computed on the host once per device.
inline cudaError_t init_tables()
{
    static uint64_t lo_f[1 << 13], hi_f[1 << 13], lo_i[1 << 13], hi_i[1 << 13];
    static uint64_t sh_lo[1 << 12], sh_hi[1 << 14], sh_lo_n[(NTT_TWLG + 1) << 12];
    static uint64_t w4096_f[4096], w4096_i[4096];
    static bool ready = false;
    if (!ready) {
        const uint64_t W = glh::root_of_unity(NTT_TWLG), Wi = glh::inv(W);
        const uint64_t W13 = glh::pow(W, 1 << 13), W13i = glh::pow(Wi, 1 << 13);
        lo_f[0] = lo_i[0] = hi_f[0] = hi_i[0] = 1;
        for (int j = 1; j < (1 << 13); j++) {
            lo_f[j] = glh::mul(lo_f[j - 1], W);
            lo_i[j] = glh::mul(lo_i[j - 1], Wi);
            hi_f[j] = glh::mul(hi_f[j - 1], W13);
            hi_i[j] = glh::mul(hi_i[j - 1], W13i);
        }
        const uint64_t s4096 = glh::pow(7, 4096);
        sh_lo[0] = sh_hi[0] = 1;
        for (int j = 1; j < (1 << 12); j++) sh_lo[j] = glh::mul(sh_lo[j - 1], 7);
        for (int j = 1; j < (1 << 14); j++) sh_hi[j] = glh::mul(sh_hi[j - 1], s4096);
        // the coset step's 1/N folded into the low table, one copy per transform size 2^lg
        const uint64_t half = glh::inv(2);
        uint64_t ninv = 1;
        for (int lg = 0; lg <= NTT_TWLG; lg++, ninv = glh::mul(ninv, half))
            for (int j = 0; j < (1 << 12); j++) sh_lo_n[(lg << 12) + j] = glh::mul(sh_lo[j], ninv);
        const uint64_t w4096 = glh::root_of_unity(12), w4096i = glh::inv(w4096);
        w4096_f[0] = w4096_i[0] = 1;
        for (int j = 1; j < 4096; j++) {
            w4096_f[j] = glh::mul(w4096_f[j - 1], w4096);
            w4096_i[j] = glh::mul(w4096_i[j - 1], w4096i);
        }
        ready = true;
    }
    cudaError_t e;
    if ((e = cudaMemcpyToSymbol(g_ntt_tw_lo_fwd, lo_f, sizeof(lo_f))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_tw_hi_fwd, hi_f, sizeof(hi_f))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_tw_lo_inv, lo_i, sizeof(lo_i))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_tw_hi_inv, hi_i, sizeof(hi_i))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_sh_lo_n, sh_lo_n, sizeof(sh_lo_n))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_sh_hi, sh_hi, sizeof(sh_hi))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_w4096_fwd, w4096_f, sizeof(w4096_f))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_w4096_inv, w4096_i, sizeof(w4096_i))) != cudaSuccess) return e;
    return cudaSuccess;
}

}  // namespace ntt
