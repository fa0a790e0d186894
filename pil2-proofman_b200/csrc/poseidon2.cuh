// Poseidon2 over Goldilocks, widths 8 / 12 / 16.
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

// ---------------------------------------------------------------------------------
// The permutation keeps each thread's W state words in shared memory at st[i*TPB] (TPB
// threads interleaved: a warp touches 32 consecutive words, no bank conflicts) and runs
// the rounds as short loops over groups of four words.  A fully unrolled register-state
// version is ~27k instructions of straight-line code, far larger than the instruction
// cache: its warps stalled on instruction fetch and it ran 1.3x slower.  (Holding a CTA's
// warps together with a barrier per round was measured too and gave nothing.)
// ---------------------------------------------------------------------------------

template <int W, int TPB>
__device__ __forceinline__ void external_layer_smem(uint64_t *st)
{
    gl::Acc s0 = {0, 0, 0}, s1 = {0, 0, 0}, s2 = {0, 0, 0}, s3 = {0, 0, 0};
#pragma unroll 1
    for (int q = 0; q < W; q += 4) {
        gl::Acc y0, y1, y2, y3;
        m4(st[(q + 0) * TPB], st[(q + 1) * TPB], st[(q + 2) * TPB], st[(q + 3) * TPB], y0, y1, y2, y3);
        s0 = gl::acc_add(s0, y0);
        s1 = gl::acc_add(s1, y1);
        s2 = gl::acc_add(s2, y2);
        s3 = gl::acc_add(s3, y3);
        st[(q + 0) * TPB] = gl::acc_reduce(y0);
        st[(q + 1) * TPB] = gl::acc_reduce(y1);
        st[(q + 2) * TPB] = gl::acc_reduce(y2);
        st[(q + 3) * TPB] = gl::acc_reduce(y3);
    }
    const uint64_t t0 = gl::acc_reduce(s0), t1 = gl::acc_reduce(s1), t2 = gl::acc_reduce(s2),
                   t3 = gl::acc_reduce(s3);
#pragma unroll 1
    for (int q = 0; q < W; q += 4) {
        st[(q + 0) * TPB] = gl::acc_reduce(gl::acc_add6464(st[(q + 0) * TPB], t0));
        st[(q + 1) * TPB] = gl::acc_reduce(gl::acc_add6464(st[(q + 1) * TPB], t1));
        st[(q + 2) * TPB] = gl::acc_reduce(gl::acc_add6464(st[(q + 2) * TPB], t2));
        st[(q + 3) * TPB] = gl::acc_reduce(gl::acc_add6464(st[(q + 3) * TPB], t3));
    }
}

template <int W, int TPB>
__device__ __forceinline__ void permute_smem(uint64_t *st)
{
    const uint64_t *C = Tab<W>::C();
    const uint64_t *D = Tab<W>::D();
#pragma unroll 1
    for (int r = 0; r <= 8; r++) {
        if (r > 0) {
            const uint64_t *Cr = C + (r <= 4 ? (r - 1) * W : 4 * W + NPARTIAL + (r - 5) * W);
#pragma unroll 1
            for (int q = 0; q < W; q += 4) {
                uint64_t a = st[(q + 0) * TPB], b = st[(q + 1) * TPB], c = st[(q + 2) * TPB], d = st[(q + 3) * TPB];
                a = gl::pow7(gl::add_c(a, Cr[q + 0]));
                b = gl::pow7(gl::add_c(b, Cr[q + 1]));
                c = gl::pow7(gl::add_c(c, Cr[q + 2]));
                d = gl::pow7(gl::add_c(d, Cr[q + 3]));
                st[(q + 0) * TPB] = a;
                st[(q + 1) * TPB] = b;
                st[(q + 2) * TPB] = c;
                st[(q + 3) * TPB] = d;
            }
        }
        external_layer_smem<W, TPB>(st);
        if (r == 4) {
            // partial rounds: x0 stays in a register; the other words stream through smem
            uint64_t x0 = st[0];
#pragma unroll 1
            for (int pr = 0; pr < NPARTIAL; pr++) {
                x0 = gl::pow7(gl::add_c(x0, C[4 * W + pr]));
                gl::Acc s = gl::acc(x0);
#pragma unroll 1
                for (int q = 4; q < W + 4; q += 4) {
                    const int i = q - 4;
                    if (i) s = gl::acc_add64(s, st[(i + 0) * TPB]);
                    s = gl::acc_add64(s, st[(i + 1) * TPB]);
                    s = gl::acc_add64(s, st[(i + 2) * TPB]);
                    s = gl::acc_add64(s, st[(i + 3) * TPB]);
                }
                const uint64_t sum = gl::acc_reduce(s);
                x0 = gl::mul_add(x0, D[0], sum);
                st[1 * TPB] = gl::mul_add(st[1 * TPB], D[1], sum);
                st[2 * TPB] = gl::mul_add(st[2 * TPB], D[2], sum);
                st[3 * TPB] = gl::mul_add(st[3 * TPB], D[3], sum);
#pragma unroll 1
                for (int q = 4; q < W; q += 4) {
                    const uint64_t a = gl::mul_add(st[(q + 0) * TPB], D[q + 0], sum);
                    const uint64_t b = gl::mul_add(st[(q + 1) * TPB], D[q + 1], sum);
                    const uint64_t c = gl::mul_add(st[(q + 2) * TPB], D[q + 2], sum);
                    const uint64_t d = gl::mul_add(st[(q + 3) * TPB], D[q + 3], sum);
                    st[(q + 0) * TPB] = a;
                    st[(q + 1) * TPB] = b;
                    st[(q + 2) * TPB] = c;
                    st[(q + 3) * TPB] = d;
                }
            }
            st[0] = x0;
        }
    }
}

}  // namespace p2
