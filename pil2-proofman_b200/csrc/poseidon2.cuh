// Poseidon2 over Goldilocks, widths 8 / 12 / 16, register-resident state.
//
// Round structure (poseidon2_goldilocks.cpp:9-41): initial external layer M_E, 4 full
// rounds (add C, x^7 on every word, M_E), 22 partial rounds (x0 += c, x0 = x0^7,
// x_i = x_i*D_i + sum(x)), 4 full rounds.  M_E is the 4x4 block M4 on every group of
// four words followed by adding the four column sums (poseidon2_goldilocks.hpp:201-240).
//
// The linear layers run on 96-bit accumulators (all coefficients are small and
// positive, so a row of M_E is below 80 * 2^64) and are reduced once per output word;
// the partial-round update x_i*D_i + sum is one 128-bit multiply-add and one reduction.
// All state words are loose (< 2^64, congruent mod p); the round constants are canonical.
#pragma once
#include "gl64.cuh"
#include "poseidon2_constants.h"

__constant__ uint64_t c_p2_C8[P2_NC_8] = {P2_C8_LIST};
__constant__ uint64_t c_p2_D8[8] = {P2_D8_LIST};
__constant__ uint64_t c_p2_C12[P2_NC_12] = {P2_C12_LIST};
__constant__ uint64_t c_p2_D12[12] = {P2_D12_LIST};
__constant__ uint64_t c_p2_C16[P2_NC_16] = {P2_C16_LIST};
__constant__ uint64_t c_p2_D16[16] = {P2_D16_LIST};

namespace p2 {

template <int W> struct Tab;
template <> struct Tab<8> {
    static __device__ __forceinline__ const uint64_t *C() { return c_p2_C8; }
    static __device__ __forceinline__ const uint64_t *D() { return c_p2_D8; }
};
template <> struct Tab<12> {
    static __device__ __forceinline__ const uint64_t *C() { return c_p2_C12; }
    static __device__ __forceinline__ const uint64_t *D() { return c_p2_D12; }
};
template <> struct Tab<16> {
    static __device__ __forceinline__ const uint64_t *C() { return c_p2_C16; }
    static __device__ __forceinline__ const uint64_t *D() { return c_p2_D16; }
};

constexpr int NPARTIAL = 22;

// M4 = [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]] on loose inputs, 96-bit outputs (< 16 * 2^64)
__device__ __forceinline__ void m4(uint64_t a, uint64_t b, uint64_t c, uint64_t d, gl::Acc &y0, gl::Acc &y1,
                                   gl::Acc &y2, gl::Acc &y3)
{
    gl::Acc ab = gl::acc_add6464(a, b);
    gl::Acc cd = gl::acc_add6464(c, d);
    gl::Acc bbcd = gl::acc_add(gl::acc_add6464(b, b), cd);  // 2b + c + d
    gl::Acc ddab = gl::acc_add(gl::acc_add6464(d, d), ab);  // a + b + 2d
    gl::Acc cd2 = gl::acc_add(cd, cd);
    gl::Acc ab2 = gl::acc_add(ab, ab);
    gl::Acc r3 = gl::acc_add(gl::acc_add(cd2, cd2), ddab);  // a + b + 4c + 6d
    gl::Acc r1 = gl::acc_add(gl::acc_add(ab2, ab2), bbcd);  // 4a + 6b + c + d
    y0 = gl::acc_add(ddab, r1);                             // 5a + 7b + c + 3d
    y1 = r1;
    y2 = gl::acc_add(bbcd, r3);                             // a + 3b + 5c + 7d
    y3 = r3;
}

template <int W>
__device__ __forceinline__ void external_layer(uint64_t (&x)[W])
{
    gl::Acc y[W];
#pragma unroll
    for (int i = 0; i < W; i += 4) m4(x[i], x[i + 1], x[i + 2], x[i + 3], y[i], y[i + 1], y[i + 2], y[i + 3]);
    gl::Acc s[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        s[j] = y[j];
#pragma unroll
        for (int i = 4 + j; i < W; i += 4) s[j] = gl::acc_add(s[j], y[i]);
    }
#pragma unroll
    for (int i = 0; i < W; i++) x[i] = gl::acc_reduce(gl::acc_add(y[i], s[i & 3]));
}

template <int W>
__device__ __forceinline__ void full_round(uint64_t (&x)[W], const uint64_t *C)
{
#pragma unroll
    for (int i = 0; i < W; i++) x[i] = gl::pow7(gl::add_c(x[i], C[i]));
    external_layer<W>(x);
}

template <int W>
__device__ __forceinline__ void partial_round(uint64_t (&x)[W], uint64_t c, const uint64_t *D)
{
    x[0] = gl::pow7(gl::add_c(x[0], c));
    gl::Acc s = gl::acc_add6464(x[0], x[1]);
#pragma unroll
    for (int i = 2; i < W; i++) s = gl::acc_add64(s, x[i]);
    uint64_t sum = gl::acc_reduce(s);
#pragma unroll
    for (int i = 0; i < W; i++) x[i] = gl::mul_add(x[i], D[i], sum);
}

// In-place permutation of a width-W state (poseidon2_goldilocks.cpp:9-41).
template <int W>
__device__ __forceinline__ void permute(uint64_t (&x)[W])
{
    const uint64_t *C = Tab<W>::C();
    const uint64_t *D = Tab<W>::D();
    external_layer<W>(x);
#pragma unroll 1
    for (int r = 0; r < 4; r++) full_round<W>(x, C + r * W);
#pragma unroll 1
    for (int r = 0; r < NPARTIAL; r++) partial_round<W>(x, C[4 * W + r], D);
#pragma unroll 1
    for (int r = 0; r < 4; r++) full_round<W>(x, C + 4 * W + NPARTIAL + r * W);
}

}  // namespace p2
