// Goldilocks field GF(p), p = 2^64 - 2^32 + 1, for sm_100a.
//
// Elements are plain uint64_t.  Device arithmetic keeps them "loose": any value in
// [0, 2^64) stands for itself mod p, the way the reference's GPU build keeps them
// partially reduced (GL64_PARTIALLY_REDUCED, goldilocks/Makefile:134).  Canonical
// form (x mod p) is produced only where values leave the library (gl_canon).
//
// The 64x64 product is the compiler's 128-bit multiply, squares take three 32x32->64
// multiply-adds (IMAD.WIDE), and both are reduced with 2^64 = 2^32 - 1 and 2^96 = -1 (mod p).
// Reference semantics: goldilocks_base_field_scalar.hpp:16-41 (add/sub), :229-258 (mul).
#pragma once
#include <stdint.h>

#define GL_P 0xFFFFFFFF00000001ULL
#define GL_EPS 0x00000000FFFFFFFFULL  // 2^64 mod p

namespace gl {

__device__ __forceinline__ uint32_t lo32(uint64_t x) { return (uint32_t)x; }
__device__ __forceinline__ uint32_t hi32(uint64_t x) { return (uint32_t)(x >> 32); }
__device__ __forceinline__ uint64_t mk64(uint32_t lo, uint32_t hi) { return ((uint64_t)hi << 32) | lo; }

// canonical representative: a - p = a + 2^32 - 1 (mod 2^64), and that sum carries out of 2^64
// exactly when a >= p, so the carry selects it.  Against the compare-subtract-select form this is
// two fewer ALU operations; the NTT butterflies canonicalise one operand each, and the LDE of
// 2^19 x 256 columns went 7.87 -> 7.47 ms with it (B200).
__device__ __forceinline__ uint64_t canon(uint64_t a)
{
    uint32_t t0, t1, k;
    asm("add.cc.u32  %0, %3, 0xffffffff;\n\t"
        "addc.cc.u32 %1, %4, 0;\n\t"
        "addc.u32    %2, 0, 0;\n\t"
        : "=r"(t0), "=r"(t1), "=r"(k)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)));
    return k ? (((uint64_t)t1 << 32) | t0) : a;
}

// Reduce the 128-bit value (r3:r2:r1:r0) to a loose 64-bit representative:
//   x = lo + hl*2^64 + hh*2^96 = lo + hl*(2^32-1) - hh  (mod p),
// where lo = r1:r0, hl = r2, hh = r3.  The signed carry c in {-1,0,1} of that sum is
// folded back as c*(2^32-1) (two's complement: +EPS or +p), which cannot wrap again.
__device__ __forceinline__ uint64_t reduce128(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3)
{
    uint32_t z0, z1, c, t0, t1;
    asm("mad.lo.cc.u32  %0, %5, 0xffffffff, %3;\n\t"
        "madc.hi.cc.u32 %1, %5, 0xffffffff, %4;\n\t"
        "addc.u32       %2, 0, 0;\n\t"
        "sub.cc.u32     %0, %0, %6;\n\t"
        "subc.cc.u32    %1, %1, 0;\n\t"
        "subc.u32       %2, %2, 0;\n\t"
        : "=r"(z0), "=r"(z1), "=r"(c)
        : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
    t0 = 0u - c;                    // c=1 -> 0xffffffff, c=-1 -> 1, c=0 -> 0
    t1 = (uint32_t)((int32_t)c >> 31);  // c=-1 -> 0xffffffff
    asm("add.cc.u32 %0, %0, %2;\n\t"
        "addc.u32   %1, %1, %3;\n\t"
        : "+r"(z0), "+r"(z1)
        : "r"(t0), "r"(t1));
    return mk64(z0, z1);
}

// Full 128-bit product (r3:r2:r1:r0): the compiler's 64x64->128 multiply of unsigned __int128.
// Over a Poseidon2 permutation it measured 8-11 % faster than the hand-written form (four
// 32x32->64 multiply-adds, each folding the previous carry word) this file used before.
__device__ __forceinline__ void mul128(uint64_t a, uint64_t b, uint32_t &r0, uint32_t &r1, uint32_t &r2,
                                       uint32_t &r3)
{
    const unsigned __int128 p = (unsigned __int128)a * b;
    const uint64_t lo = (uint64_t)p, hi = (uint64_t)(p >> 64);
    r0 = lo32(lo);
    r1 = hi32(lo);
    r2 = lo32(hi);
    r3 = hi32(hi);
}

// a^2 = a0^2 + 2*a0*a1*2^32 + a1^2*2^64 with three wide products.
__device__ __forceinline__ void sqr128(uint64_t a, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    const uint32_t a0 = lo32(a), a1 = hi32(a);
    uint64_t p00, c, w;
    asm("mul.wide.u32 %0, %1, %2;" : "=l"(p00) : "r"(a0), "r"(a0));
    asm("mul.wide.u32 %0, %1, %2;" : "=l"(c) : "r"(a0), "r"(a1));
    // 2c = (cb : c2hi : c2lo)
    const uint32_t c2lo = lo32(c) << 1, c2hi = __funnelshift_l(lo32(c), hi32(c), 1), cb = hi32(c) >> 31;
    uint32_t s1, ad0, ad1;
    asm("add.cc.u32  %0, %3, %4;\n\t"
        "addc.cc.u32 %1, %5, 0;\n\t"
        "addc.u32    %2, %6, 0;\n\t"
        : "=r"(s1), "=r"(ad0), "=r"(ad1)
        : "r"(hi32(p00)), "r"(c2lo), "r"(c2hi), "r"(cb));
    asm("mad.wide.u32 %0, %1, %1, %2;" : "=l"(w) : "r"(a1), "l"(mk64(ad0, ad1)));
    r0 = lo32(p00);
    r1 = s1;
    r2 = lo32(w);
    r3 = hi32(w);
}

__device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b)
{
    uint32_t r0, r1, r2, r3;
    mul128(a, b, r0, r1, r2, r3);
    return reduce128(r0, r1, r2, r3);
}

// a*b + c as one 128-bit value, one reduction ((2^64-1)^2 + 2^64-1 < 2^128)
__device__ __forceinline__ uint64_t mul_add(uint64_t a, uint64_t b, uint64_t c)
{
    const unsigned __int128 v = (unsigned __int128)a * b + c;
    const uint64_t lo = (uint64_t)v, hi = (uint64_t)(v >> 64);
    return reduce128(lo32(lo), hi32(lo), lo32(hi), hi32(hi));
}

__device__ __forceinline__ uint64_t sqr(uint64_t a)
{
    uint32_t r0, r1, r2, r3;
    sqr128(a, r0, r1, r2, r3);
    return reduce128(r0, r1, r2, r3);
}

// a + b for loose a and loose b: a carry out of 2^64 is worth EPS; a second carry
// (both operands near 2^64) is folded the same way and cannot repeat.
__device__ __forceinline__ uint64_t add(uint64_t a, uint64_t b)
{
    uint32_t s0, s1, c;
    asm("add.cc.u32  %0, %3, %5;\n\t"
        "addc.cc.u32 %1, %4, %6;\n\t"
        "addc.u32    %2, 0, 0;\n\t"
        : "=r"(s0), "=r"(s1), "=r"(c)
        : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)));
    uint32_t m = 0u - c;
    asm("add.cc.u32  %0, %0, %3;\n\t"
        "addc.cc.u32 %1, %1, 0;\n\t"
        "addc.u32    %2, 0, 0;\n\t"
        : "+r"(s0), "+r"(s1), "=r"(c)
        : "r"(m));
    m = 0u - c;
    asm("add.cc.u32  %0, %0, %2;\n\t"
        "addc.u32    %1, %1, 0;\n\t"
        : "+r"(s0), "+r"(s1)
        : "r"(m));
    return mk64(s0, s1);
}

// a + b where b < p (canonical): at most one carry fix-up is needed
__device__ __forceinline__ uint64_t add_c(uint64_t a, uint64_t b)
{
    uint32_t s0, s1, c;
    asm("add.cc.u32  %0, %3, %5;\n\t"
        "addc.cc.u32 %1, %4, %6;\n\t"
        "addc.u32    %2, 0, 0;\n\t"
        : "=r"(s0), "=r"(s1), "=r"(c)
        : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)));
    uint32_t m = 0u - c;
    asm("add.cc.u32  %0, %0, %2;\n\t"
        "addc.u32    %1, %1, 0;\n\t"
        : "+r"(s0), "+r"(s1)
        : "r"(m));
    return mk64(s0, s1);
}

// a - b for loose a, b: a borrow is worth -EPS; a second borrow is folded the same way.
__device__ __forceinline__ uint64_t sub(uint64_t a, uint64_t b)
{
    uint32_t s0, s1, c;
    asm("sub.cc.u32  %0, %3, %5;\n\t"
        "subc.cc.u32 %1, %4, %6;\n\t"
        "subc.u32    %2, 0, 0;\n\t"
        : "=r"(s0), "=r"(s1), "=r"(c)
        : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)));
    uint32_t m = c;  // 0 or 0xffffffff (= EPS low word)
    asm("sub.cc.u32  %0, %0, %3;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.u32    %2, 0, 0;\n\t"
        : "+r"(s0), "+r"(s1), "=r"(c)
        : "r"(m));
    m = c;
    asm("sub.cc.u32  %0, %0, %2;\n\t"
        "subc.u32    %1, %1, 0;\n\t"
        : "+r"(s0), "+r"(s1)
        : "r"(m));
    return mk64(s0, s1);
}

// a - b where b < p (canonical): one borrow fix-up suffices (a second borrow would need b > p)
__device__ __forceinline__ uint64_t sub_c(uint64_t a, uint64_t b)
{
    uint32_t s0, s1, c;
    asm("sub.cc.u32  %0, %3, %5;\n\t"
        "subc.cc.u32 %1, %4, %6;\n\t"
        "subc.u32    %2, 0, 0;\n\t"
        : "=r"(s0), "=r"(s1), "=r"(c)
        : "r"(lo32(a)), "r"(hi32(a)), "r"(lo32(b)), "r"(hi32(b)));
    asm("sub.cc.u32  %0, %0, %2;\n\t"
        "subc.u32    %1, %1, 0;\n\t"
        : "+r"(s0), "+r"(s1)
        : "r"(c));
    return mk64(s0, s1);
}

// x * 2^S mod p for 0 < S < 96 by shifts: x << S spans at most three 32-bit words placed at word
// offset S/32, folded with 2^64 = 2^32 - 1, 2^96 = -1 and 2^128 = -2^32 (mod p).  At offset 0 the
// words are (u1:u0) + u2 * 2^64: one multiply-add and one carry fold; at offset 2 they are
// u0 * 2^64 + (u2:u1) * 2^96: one product and one subtraction; offset 1 takes the general 128-bit
// reduction.  Multiplication by the radix-16 roots of unity (powers of w_16 = 2^12) thus costs
// three shifts and a short reduction instead of four wide products.
template <int S>
__device__ __forceinline__ uint64_t mul_pow2(uint64_t x)
{
    static_assert(S > 0 && S < 96, "shift out of range");
    constexpr int Q = S / 32, T = S % 32;
    const uint32_t x0 = lo32(x), x1 = hi32(x);
    uint32_t u0, u1, u2;
    if (T == 0) {
        u0 = x0;
        u1 = x1;
        u2 = 0;
    } else {
        u0 = x0 << T;
        u1 = __funnelshift_l(x0, x1, T);
        u2 = x1 >> (32 - T);
    }
    if (Q == 0) {
        // (u1:u0) + u2 * 2^64 = (u1:u0) + u2 * (2^32 - 1): one carry at most, folded as 2^32 - 1
        uint32_t z0, z1, c;
        asm("mad.lo.cc.u32  %0, %5, 0xffffffff, %3;\n\t"
            "madc.hi.cc.u32 %1, %5, 0xffffffff, %4;\n\t"
            "addc.u32       %2, 0, 0;\n\t"
            : "=r"(z0), "=r"(z1), "=r"(c)
            : "r"(u0), "r"(u1), "r"(u2));
        const uint32_t m = 0u - c;
        asm("add.cc.u32 %0, %0, %2;\n\t"
            "addc.u32   %1, %1, 0;\n\t"
            : "+r"(z0), "+r"(z1)
            : "r"(m));
        return mk64(z0, z1);
    }
    if (Q == 1) return reduce128(0u, u0, u1, u2);
    // u0 * 2^64 + u1 * 2^96 + u2 * 2^128 = u0 * (2^32 - 1) - (u2 * 2^32 + u1), and u2 < 2^T <= 2^31
    // keeps the subtrahend below p
    uint64_t w;
    asm("mul.wide.u32 %0, %1, 0xffffffff;" : "=l"(w) : "r"(u0));
    return sub_c(w, mk64(u1, u2));
}

// x^7 = x^3 * x^4, the Poseidon2 S-box (poseidon2_goldilocks.hpp:147-155)
__device__ __forceinline__ uint64_t pow7(uint64_t x)
{
    uint64_t x2 = sqr(x);
    uint64_t x3 = mul(x, x2);
    uint64_t x4 = sqr(x2);
    return mul(x3, x4);
}

// ---- accumulators for linear layers with small positive coefficients ----
// Sums of a few dozen loose words times small coefficients stay below 2^96.  They are kept as
// 128-bit integers: the compiler's carry chains for these adds measured 1.8 % faster over a
// Poseidon2 permutation than hand-written three-word add.cc chains.
struct Acc {
    unsigned __int128 v;
};

__device__ __forceinline__ Acc acc(uint64_t a) { return Acc{(unsigned __int128)a}; }
__device__ __forceinline__ Acc acc_add(Acc a, Acc b) { return Acc{a.v + b.v}; }
__device__ __forceinline__ Acc acc_add64(Acc a, uint64_t b) { return Acc{a.v + b}; }
__device__ __forceinline__ Acc acc_add6464(uint64_t a, uint64_t b) { return Acc{(unsigned __int128)a + b}; }
// lo + hi * 2^32 for lo, hi < 2^64 - 2^32 (two 64-bit sums of 32x32 products over the low and
// high halves of the inputs)
__device__ __forceinline__ Acc acc_lohi(uint64_t lo, uint64_t hi)
{
    return Acc{(unsigned __int128)lo + ((unsigned __int128)hi << 32)};
}

// fold (w2:lo) = lo + w2*2^64 = lo + w2*(2^32-1) for w2 < 2^32: a single carry may remain, worth EPS
__device__ __forceinline__ uint64_t acc_reduce(Acc a)
{
    const uint64_t lo = (uint64_t)a.v;
    const uint32_t w2 = (uint32_t)(a.v >> 64);
    uint32_t z0, z1, c;
    asm("mad.lo.cc.u32  %0, %5, 0xffffffff, %3;\n\t"
        "madc.hi.cc.u32 %1, %5, 0xffffffff, %4;\n\t"
        "addc.u32       %2, 0, 0;\n\t"
        : "=r"(z0), "=r"(z1), "=r"(c)
        : "r"(lo32(lo)), "r"(hi32(lo)), "r"(w2));
    uint32_t m = 0u - c;
    asm("add.cc.u32  %0, %0, %2;\n\t"
        "addc.u32    %1, %1, 0;\n\t"
        : "+r"(z0), "+r"(z1)
        : "r"(m));
    return mk64(z0, z1);
}

}  // namespace gl

// ---------------------------------------------------------------- host side ----
namespace glh {
static inline uint64_t canon(uint64_t a) { return a >= GL_P ? a - GL_P : a; }
static inline uint64_t mul(uint64_t a, uint64_t b)
{
    unsigned __int128 x = (unsigned __int128)a * b;
    return (uint64_t)(x % GL_P);
}
static inline uint64_t add(uint64_t a, uint64_t b)
{
    unsigned __int128 x = (unsigned __int128)a + b;
    return (uint64_t)(x % GL_P);
}
static inline uint64_t pow(uint64_t b, uint64_t e)
{
    uint64_t acc = 1;
    b = canon(b);
    while (e) {
        if (e & 1) acc = mul(acc, b);
        b = mul(b, b);
        e >>= 1;
    }
    return acc;
}
static inline uint64_t inv(uint64_t a) { return pow(a, GL_P - 2); }
// W[k]: the reference's 2^k-th roots of unity (goldilocks_base_field.cpp:11-44), which are
// W[32] = 0x64fdd1a46201e246 squared down: W[k] = W[k+1]^2.
static inline uint64_t root_of_unity(unsigned k)
{
    uint64_t w = 0x64fdd1a46201e246ULL;
    for (unsigned i = 32; i > k; i--) w = mul(w, w);
    return w;
}
}  // namespace glh
