// Poseidon1 over Goldilocks (hash family 1), widths 8 / 12 / 16.
//
// The reference's optimised round structure (poseidon_goldilocks.cpp:13-51): add C_0; three
// full rounds (x^7, add the next round's constants, state <- M^T x); x^7, add C_4, state <- P^T x;
// 22 sparse partial rounds (x0 <- x0^7 + c_r; x0' = <x, S_r[0..W)>; x_i += x0 * S_r[W-1+i] for
// i >= 1); three full rounds with M; x^7 and M.  mvp_ (poseidon_goldilocks.hpp:210-224) applies
// its matrix transposed: out_i = sum_j mat[j][i] * x_j.
//
// Arithmetic:
//   * M has entries below 2^7, so each output of M^T x is two sums of (32-bit half of x_j) x
//     (entry): integers below 2^41, which the FP64 pipe computes exactly (fused multiply-adds
//     on doubles; in and out by exponent-bias bit patterns, no conversion instructions).  They
//     are combined into a 96-bit value and folded once.  On the IMAD pipe the same products
//     were 37 % of the permutation's wide multiplies; on the otherwise idle FP64 pipe the W16
//     permutation runs 12.5 % faster (B200, same outputs).
//   * P and the partial-round vectors S are full field elements: the dot products accumulate
//     128-bit products in 160 bits and reduce once (2^128 = -2^32 mod p).
// State in shared memory, word i of this thread at st[i*TPB], like the Poseidon2 kernels; the
// matrix steps write to a second W x TPB area and copy back.
#pragma once
#include "gl64.cuh"
#include "poseidon1_constants.h"

__constant__ uint64_t c_p1_C8[P1_NC_8] = {P1_C8_LIST};
__constant__ uint64_t c_p1_M8[64] = {P1_M8_LIST};
__constant__ uint64_t c_p1_P8[64] = {P1_P8_LIST};
__constant__ uint64_t c_p1_S8[P1_NS_8] = {P1_S8_LIST};
__constant__ uint64_t c_p1_C12[P1_NC_12] = {P1_C12_LIST};
__constant__ uint64_t c_p1_M12[144] = {P1_M12_LIST};
__constant__ uint64_t c_p1_P12[144] = {P1_P12_LIST};
__constant__ uint64_t c_p1_S12[P1_NS_12] = {P1_S12_LIST};
__constant__ uint64_t c_p1_C16[P1_NC_16] = {P1_C16_LIST};
__constant__ uint64_t c_p1_M16[256] = {P1_M16_LIST};
__constant__ uint64_t c_p1_P16[256] = {P1_P16_LIST};
__constant__ uint64_t c_p1_S16[P1_NS_16] = {P1_S16_LIST};

__constant__ double c_p1_Md8[64] = {P1_M8_LIST};
__constant__ double c_p1_Md12[144] = {P1_M12_LIST};
__constant__ double c_p1_Md16[256] = {P1_M16_LIST};

namespace p1 {

template <int W> struct Tab;
template <> struct Tab<8> {
    static __device__ __forceinline__ const double *Md() { return c_p1_Md8; }
    static __device__ __forceinline__ const uint64_t *C() { return c_p1_C8; }
    static __device__ __forceinline__ const uint64_t *M() { return c_p1_M8; }
    static __device__ __forceinline__ const uint64_t *P() { return c_p1_P8; }
    static __device__ __forceinline__ const uint64_t *S() { return c_p1_S8; }
};
template <> struct Tab<12> {
    static __device__ __forceinline__ const double *Md() { return c_p1_Md12; }
    static __device__ __forceinline__ const uint64_t *C() { return c_p1_C12; }
    static __device__ __forceinline__ const uint64_t *M() { return c_p1_M12; }
    static __device__ __forceinline__ const uint64_t *P() { return c_p1_P12; }
    static __device__ __forceinline__ const uint64_t *S() { return c_p1_S12; }
};
template <> struct Tab<16> {
    static __device__ __forceinline__ const double *Md() { return c_p1_Md16; }
    static __device__ __forceinline__ const uint64_t *C() { return c_p1_C16; }
    static __device__ __forceinline__ const uint64_t *M() { return c_p1_M16; }
    static __device__ __forceinline__ const uint64_t *P() { return c_p1_P16; }
    static __device__ __forceinline__ const uint64_t *S() { return c_p1_S16; }
};

constexpr int NPARTIAL = P1_NPARTIAL;

// 160-bit accumulator of 128-bit products
struct Acc160 {
    uint32_t w[5];
};

__device__ __forceinline__ void acc160_mul_add(Acc160 &a, uint64_t x, uint64_t y)
{
    uint32_t r0, r1, r2, r3;
    gl::mul128(x, y, r0, r1, r2, r3);
    asm("add.cc.u32  %0, %0, %5;\n\t"
        "addc.cc.u32 %1, %1, %6;\n\t"
        "addc.cc.u32 %2, %2, %7;\n\t"
        "addc.cc.u32 %3, %3, %8;\n\t"
        "addc.u32    %4, %4, 0;\n\t"
        : "+r"(a.w[0]), "+r"(a.w[1]), "+r"(a.w[2]), "+r"(a.w[3]), "+r"(a.w[4])
        : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
}

// x = A + w4 * 2^128 with 2^128 = -2^32 (mod p): reduce A, then subtract w4 * 2^32 (< p)
__device__ __forceinline__ uint64_t acc160_reduce(const Acc160 &a)
{
    const uint64_t y = gl::reduce128(a.w[0], a.w[1], a.w[2], a.w[3]);
    return gl::sub(y, (uint64_t)a.w[4] << 32);
}

// exact u32 -> double: the double 2^52 + u (exponent bias bits over u) minus 2^52
__device__ __forceinline__ double u32_f64(uint32_t u) { return __hiloint2double(0x43300000, (int)u) - 4503599627370496.0; }
// integer-valued double 0 <= v < 2^52 -> its value: the mantissa bits of v + 2^52
__device__ __forceinline__ uint64_t f64_u52(double v)
{
    return (uint64_t)__double_as_longlong(v + 4503599627370496.0) & 0xFFFFFFFFFFFFFull;
}

// out_i = sum_j M[j][i] x_j for the small-entry MDS matrix, on the FP64 pipe: every partial sum
// of the 32-bit halves times entries < 2^7 is an integer below 2^41, exact in a double.  Passes
// of four outputs (their two sums in registers), inputs re-read and converted per pass.
template <int W, int TPB>
__device__ __forceinline__ void mvp_small(uint64_t *st, uint64_t *tmp)
{
    const double *M = Tab<W>::Md();
    constexpr int PASS = 4;  // outputs per pass
#pragma unroll
    for (int i0 = 0; i0 < W; i0 += PASS) {
        double L[PASS], H[PASS];
#pragma unroll
        for (int u = 0; u < PASS; u++) L[u] = H[u] = 0.0;
#pragma unroll
        for (int j = 0; j < W; j++) {
            const uint64_t x = st[j * TPB];
            const double xl = u32_f64(gl::lo32(x)), xh = u32_f64(gl::hi32(x));
#pragma unroll
            for (int u = 0; u < PASS; u++) {
                const double m = M[j * W + i0 + u];
                L[u] = fma(m, xl, L[u]);
                H[u] = fma(m, xh, H[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < PASS; u++) {
            // l + h * 2^32 (l, h < 2^41)
            tmp[(i0 + u) * TPB] = gl::acc_reduce(gl::acc_lohi(f64_u52(L[u]), f64_u52(H[u])));
        }
        asm volatile("" ::: "memory");  // keep the next pass's loads after this pass's stores
    }
#pragma unroll
    for (int i = 0; i < W; i++) st[i * TPB] = tmp[i * TPB];
}

// out_i = sum_j P[j][i] x_j for a matrix of full field elements
template <int W, int TPB>
__device__ __forceinline__ void mvp_full(uint64_t *st, uint64_t *tmp, const uint64_t *P)
{
#pragma unroll 1
    for (int i0 = 0; i0 < W; i0 += 2) {
        Acc160 a0 = {{0, 0, 0, 0, 0}}, a1 = {{0, 0, 0, 0, 0}};
#pragma unroll 4
        for (int j = 0; j < W; j++) {
            const uint64_t x = st[j * TPB];
            acc160_mul_add(a0, x, P[j * W + i0]);
            acc160_mul_add(a1, x, P[j * W + i0 + 1]);
        }
        tmp[i0 * TPB] = acc160_reduce(a0);
        tmp[(i0 + 1) * TPB] = acc160_reduce(a1);
    }
#pragma unroll
    for (int i = 0; i < W; i++) st[i * TPB] = tmp[i * TPB];
}

// x^7 then + c (c canonical) on every word
template <int W, int TPB>
__device__ __forceinline__ void sbox_add(uint64_t *st, const uint64_t *c)
{
#pragma unroll 1
    for (int q = 0; q < W; q += 4) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t x = gl::pow7(st[(q + u) * TPB]);
            st[(q + u) * TPB] = c ? gl::add_c(x, c[q + u]) : x;
        }
    }
}

// The permutation of the thread's state st[i*TPB] (loose words in, loose words out);
// tmp: a second W x TPB area of the thread.  The eight full rounds run as one loop (round 3
// applies P instead of M, the partial rounds sit between rounds 3 and 4, the last round adds no
// constants) so the S-box and matrix code appears once: unrolled copies overflowed the
// instruction cache.
template <int W, int TPB>
__device__ __forceinline__ void permute_smem(uint64_t *st, uint64_t *tmp)
{
    const uint64_t *C = Tab<W>::C();
    const uint64_t *S = Tab<W>::S();
#pragma unroll
    for (int i = 0; i < W; i++) st[i * TPB] = gl::add_c(st[i * TPB], C[i]);
#pragma unroll 1
    for (int r = 0; r < 8; r++) {
        if (r == 4) {
            uint64_t x0 = st[0];
#pragma unroll 1
            for (int pr = 0; pr < NPARTIAL; pr++) {
                const uint64_t *Sr = S + (2 * W - 1) * pr;
                x0 = gl::add_c(gl::pow7(x0), C[5 * W + pr]);
                Acc160 a = {{0, 0, 0, 0, 0}};
                acc160_mul_add(a, x0, Sr[0]);
#pragma unroll 4
                for (int i = 1; i < W; i++) {
                    const uint64_t xi = st[i * TPB];
                    acc160_mul_add(a, xi, Sr[i]);
                    st[i * TPB] = gl::mul_add(x0, Sr[W - 1 + i], xi);
                }
                x0 = acc160_reduce(a);
            }
            st[0] = x0;
        }
        const uint64_t *c = r < 4 ? C + (r + 1) * W : (r < 7 ? C + 5 * W + NPARTIAL + (r - 4) * W : nullptr);
        sbox_add<W, TPB>(st, c);
        if (r == 3)
            mvp_full<W, TPB>(st, tmp, Tab<W>::P());
        else
            mvp_small<W, TPB>(st, tmp);
    }
}

}  // namespace p1
