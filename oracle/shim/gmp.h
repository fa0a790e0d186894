/* Minimal GMP stand-in for compiling the reference's Goldilocks CPU sources
 * (goldilocks_base_field.cpp, ntt_goldilocks.cpp, poseidon2_goldilocks.cpp)
 * where only the GMP runtime library, not its headers, is installed.
 *
 * Test infrastructure only: it backs the reference CPU build under oracle/_ref.
 * Values are held in a signed 128-bit integer.  That covers every use on the
 * commit path: string/scalar conversion of field elements (< 2^65 in flight,
 * goldilocks_base_field_tools.hpp:72-186) and the NTT constructor's 2-adicity,
 * non-residue and 2^-1 set-up modulo p < 2^64 (ntt_goldilocks.hpp:78-161).
 */
#ifndef ORACLE_SHIM_GMP_H
#define ORACLE_SHIM_GMP_H

#include <stddef.h>
#include <stdint.h>
#include <string.h>

typedef struct {
    __int128 v;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;

static inline void mpz_init(mpz_ptr x) { x->v = 0; }
static inline void mpz_clear(mpz_ptr x) { (void)x; }
static inline void mpz_set(mpz_ptr r, mpz_srcptr a) { r->v = a->v; }
static inline void mpz_set_ui(mpz_ptr r, unsigned long a) { r->v = (__int128)a; }
static inline void mpz_set_si(mpz_ptr r, long a) { r->v = (__int128)a; }
static inline void mpz_add_ui(mpz_ptr r, mpz_srcptr a, unsigned long b) { r->v = a->v + (__int128)b; }
static inline void mpz_sub_ui(mpz_ptr r, mpz_srcptr a, unsigned long b) { r->v = a->v - (__int128)b; }
/* floor division by 2^b: an arithmetic right shift floors for negatives too */
static inline void mpz_fdiv_q_2exp(mpz_ptr r, mpz_srcptr a, unsigned long b) { r->v = a->v >> b; }
static inline int mpz_cmp_ui(mpz_srcptr a, unsigned long b)
{
    __int128 bb = (__int128)b;
    return a->v < bb ? -1 : (a->v > bb ? 1 : 0);
}
static inline int mpz_cmp(mpz_srcptr a, mpz_srcptr b) { return a->v < b->v ? -1 : (a->v > b->v ? 1 : 0); }
static inline int mpz_tstbit(mpz_srcptr a, unsigned long bit) { return (int)((a->v >> bit) & 1); }
static inline unsigned long mpz_get_ui(mpz_srcptr a) { return (unsigned long)(unsigned __int128)a->v; }
static inline long mpz_get_si(mpz_srcptr a) { return (long)a->v; }

/* |a| mod m for 0 <= a, 0 < m < 2^64 */
static inline unsigned __int128 shim_mod(__int128 a, __int128 m)
{
    __int128 r = a % m;
    if (r < 0) r += m;
    return (unsigned __int128)r;
}

static inline void mpz_powm(mpz_ptr r, mpz_srcptr base, mpz_srcptr exp, mpz_srcptr mod)
{
    unsigned __int128 m = (unsigned __int128)mod->v;
    unsigned __int128 b = shim_mod(base->v, mod->v);
    unsigned __int128 e = (unsigned __int128)exp->v;
    unsigned __int128 acc = 1 % m;
    while (e) {
        if (e & 1) acc = (acc * b) % m; /* operands < 2^64: product fits */
        b = (b * b) % m;
        e >>= 1;
    }
    r->v = (__int128)acc;
}

/* modular inverse by the extended Euclidean algorithm; returns 0 if none */
static inline int mpz_invert(mpz_ptr r, mpz_srcptr a, mpz_srcptr mod)
{
    __int128 m = mod->v;
    __int128 t = 0, newt = 1;
    __int128 rr = m, newr = (__int128)shim_mod(a->v, m);
    while (newr != 0) {
        __int128 q = rr / newr;
        __int128 tmp = t - q * newt;
        t = newt;
        newt = tmp;
        tmp = rr - q * newr;
        rr = newr;
        newr = tmp;
    }
    if (rr != 1) return 0;
    if (t < 0) t += m;
    r->v = t;
    return 1;
}

/* Only the single-word import used by the reference (count 1, size 8). */
static inline void mpz_import(mpz_ptr rop, size_t count, int order, size_t size, int endian, size_t nails,
                              const void *op)
{
    (void)order;
    (void)endian;
    (void)nails;
    unsigned __int128 v = 0;
    if (count == 1 && size == 8) {
        uint64_t w;
        memcpy(&w, op, 8);
        v = w;
    } else if (count == 1 && size == 4) {
        uint32_t w;
        memcpy(&w, op, 4);
        v = w;
    }
    rop->v = (__int128)v;
}

#endif
