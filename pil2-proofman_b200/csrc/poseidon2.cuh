// Poseidon2 over Goldilocks, widths 8 / 12 / 16.
//
// Round structure (poseidon2_goldilocks.cpp:9-41): initial external layer M_E, 4 full
// rounds (add C, x^7 on every word, M_E), 22 partial rounds (x0 += c, x0 = x0^7,
// x_i = x_i*D_i + sum(x)), 4 full rounds.  M_E is the 4x4 block M4 on every group of
// four words followed by adding the four column sums (poseidon2_goldilocks.hpp:201-240).
//
// The linear layers run on 96-bit accumulators (all coefficients are small and
// positive) and are reduced once per output word: by linearity M_E x = M4(block) + M4(S)
// with S the column sums of the blocks (M4(S) taken on the unreduced 96-bit sums), so each
// output is M4(block) + M4(S) (+ the next full round's constants, folded in before the
// reduction) < 81 * 2^64.  The partial-round
// update x_i*D_i + sum is one 128-bit multiply-add and one reduction, and the next round's sum
// of x_1.. is accumulated while they are updated.  Against the form that reduced M4(block)
// first, added the reduced column sums and reduced again, and re-read x_1.. for every partial
// round's sum, this is 6 % more W16 permutations per second (B200).
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

// M4 on 96-bit inputs (each below 2^92): 96-bit outputs (coefficient sums <= 16)
__device__ __forceinline__ void m4_acc(gl::Acc a, gl::Acc b, gl::Acc c, gl::Acc d, gl::Acc &y0, gl::Acc &y1,
                                       gl::Acc &y2, gl::Acc &y3)
{
    gl::Acc ab = gl::acc_add(a, b);
    gl::Acc cd = gl::acc_add(c, d);
    gl::Acc bbcd = gl::acc_add(gl::acc_add(b, b), cd);
    gl::Acc ddab = gl::acc_add(gl::acc_add(d, d), ab);
    gl::Acc cd2 = gl::acc_add(cd, cd);
    gl::Acc ab2 = gl::acc_add(ab, ab);
    gl::Acc r3 = gl::acc_add(gl::acc_add(cd2, cd2), ddab);
    gl::Acc r1 = gl::acc_add(gl::acc_add(ab2, ab2), bbcd);
    y0 = gl::acc_add(ddab, r1);
    y1 = r1;
    y2 = gl::acc_add(bbcd, r3);
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

// M_E x = M4(block) + M4(sum of the blocks) (linearity), plus the next round's constants cn
// (canonical; null: none) before the single reduction of each output.
template <int W, int TPB>
__device__ __forceinline__ void external_layer_smem(uint64_t *st, const uint64_t *cn)
{
    gl::Acc S0 = gl::acc_add6464(st[0 * TPB], st[4 * TPB]), S1 = gl::acc_add6464(st[1 * TPB], st[5 * TPB]),
            S2 = gl::acc_add6464(st[2 * TPB], st[6 * TPB]), S3 = gl::acc_add6464(st[3 * TPB], st[7 * TPB]);
#pragma unroll
    for (int q = 8; q < W; q += 4) {
        S0 = gl::acc_add64(S0, st[(q + 0) * TPB]);
        S1 = gl::acc_add64(S1, st[(q + 1) * TPB]);
        S2 = gl::acc_add64(S2, st[(q + 2) * TPB]);
        S3 = gl::acc_add64(S3, st[(q + 3) * TPB]);
    }
    gl::Acc t0, t1, t2, t3;
    m4_acc(S0, S1, S2, S3, t0, t1, t2, t3);
#pragma unroll 1
    for (int q = 0; q < W; q += 4) {
        gl::Acc y0, y1, y2, y3;
        m4(st[(q + 0) * TPB], st[(q + 1) * TPB], st[(q + 2) * TPB], st[(q + 3) * TPB], y0, y1, y2, y3);
        y0 = gl::acc_add(y0, t0);
        y1 = gl::acc_add(y1, t1);
        y2 = gl::acc_add(y2, t2);
        y3 = gl::acc_add(y3, t3);
        if (cn) {
            y0 = gl::acc_add64(y0, cn[q + 0]);
            y1 = gl::acc_add64(y1, cn[q + 1]);
            y2 = gl::acc_add64(y2, cn[q + 2]);
            y3 = gl::acc_add64(y3, cn[q + 3]);
        }
        st[(q + 0) * TPB] = gl::acc_reduce(y0);
        st[(q + 1) * TPB] = gl::acc_reduce(y1);
        st[(q + 2) * TPB] = gl::acc_reduce(y2);
        st[(q + 3) * TPB] = gl::acc_reduce(y3);
    }
}

// Rounds: r = 0 the initial M_E; r = 1..8 the full rounds (x^7 on every word, M_E), the 22
// partial rounds after r = 4.  Each full round's constants are added by the linear layer before
// it, except round 5's, which follows the partial rounds.
template <int W, int TPB>
__device__ __forceinline__ void permute_smem(uint64_t *st)
{
    const uint64_t *C = Tab<W>::C();
    const uint64_t *D = Tab<W>::D();
#pragma unroll 1
    for (int r = 0; r <= 8; r++) {
        if (r > 0) {
            const uint64_t *Cr = r == 5 ? C + 4 * W + NPARTIAL : nullptr;
#pragma unroll 1
            for (int q = 0; q < W; q += 4) {
                uint64_t a = st[(q + 0) * TPB], b = st[(q + 1) * TPB], c = st[(q + 2) * TPB], d = st[(q + 3) * TPB];
                if (Cr) {
                    a = gl::add_c(a, Cr[q + 0]);
                    b = gl::add_c(b, Cr[q + 1]);
                    c = gl::add_c(c, Cr[q + 2]);
                    d = gl::add_c(d, Cr[q + 3]);
                }
                st[(q + 0) * TPB] = gl::pow7(a);
                st[(q + 1) * TPB] = gl::pow7(b);
                st[(q + 2) * TPB] = gl::pow7(c);
                st[(q + 3) * TPB] = gl::pow7(d);
            }
        }
        // constants of round r + 1 (rounds 1..4: C + r * W; rounds 6..8: C + 4W + 22 + (r - 4) * W)
        const uint64_t *cn = r < 4 ? C + r * W : (r >= 5 && r < 8 ? C + 4 * W + NPARTIAL + (r - 4) * W : nullptr);
        external_layer_smem<W, TPB>(st, cn);
        if (r == 4) {
            // partial rounds: x0 in a register; the sum of x_1.. for the next round is
            // accumulated while they are updated
            uint64_t x0 = st[0];
            gl::Acc rest = gl::acc_add6464(st[1 * TPB], st[2 * TPB]);
#pragma unroll
            for (int i = 3; i < W; i++) rest = gl::acc_add64(rest, st[i * TPB]);
#pragma unroll 1
            for (int pr = 0; pr < NPARTIAL; pr++) {
                x0 = gl::pow7(gl::add_c(x0, C[4 * W + pr]));
                const uint64_t sum = gl::acc_reduce(gl::acc_add64(rest, x0));
                x0 = gl::mul_add(x0, D[0], sum);
                const uint64_t u1 = gl::mul_add(st[1 * TPB], D[1], sum);
                const uint64_t u2 = gl::mul_add(st[2 * TPB], D[2], sum);
                const uint64_t u3 = gl::mul_add(st[3 * TPB], D[3], sum);
                st[1 * TPB] = u1;
                st[2 * TPB] = u2;
                st[3 * TPB] = u3;
                rest = gl::acc_add64(gl::acc_add6464(u1, u2), u3);
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
                    rest = gl::acc_add64(gl::acc_add64(gl::acc_add64(gl::acc_add64(rest, a), b), c), d);
                }
            }
            st[0] = x0;
        }
    }
}

}  // namespace p2
