/* CPU oracle for the LDE + Poseidon2-Merkle commit path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's CPU algorithm, used by tests/ (and the
 * oracle leg of bench.py) to check the CUDA path; the product never links it.
 * Every value it returns is canonical (x mod p).  Pinned against the reference's
 * golden vectors (tests/test_oracle_golden.py) and against the reference CPU
 * sources compiled unmodified under oracle/_ref.
 *
 * Reference sections restated here (paths inside pil2-stark/src/goldilocks/src):
 *   field                goldilocks_base_field_scalar.hpp:16-41,229-258 ; p, W[], SHIFT: goldilocks_base_field.cpp:5-50
 *   LDE                  ntt_goldilocks.cpp:369-404 (INTT with r_[i] = 7^i/N, zero pad, NTT on NExt);
 *                        computeR ntt_goldilocks.hpp:48-60
 *   Poseidon2 permute    poseidon2_goldilocks.cpp:9-41 ; matmul_m4_/matmul_external_ poseidon2_goldilocks.hpp:201-240
 *   linear hash          poseidon2_goldilocks.cpp:42-77
 *   Merkle tree          poseidon2_goldilocks.cpp:129-175 ; getTreeNumElements goldilocks_tooling.hpp:9-21
 *   Poseidon1 permute    poseidon_goldilocks.cpp:13-51 ; pow7/add_/prod_/dot_/mvp_ poseidon_goldilocks.hpp:137-224
 *   Poseidon1 sponge     poseidon_goldilocks.cpp:53-89 ; tree :91-150 (node input zero-padded to W)
 *   hash family switch   utils/hash_family.hpp:45-66 (set_hash_family: 1 = Poseidon1, 2 = Poseidon2)
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "poseidon1_constants.h"
#include "poseidon2_constants.h"

#define GL_P 0xFFFFFFFF00000001ULL
#define GL_EPS 0xFFFFFFFFULL /* 2^64 mod p */

typedef unsigned __int128 u128;

static inline uint64_t canon(uint64_t a) { return a >= GL_P ? a - GL_P : a; }

static inline uint64_t gl_add(uint64_t a, uint64_t b)
{
    /* a, b canonical: a + b < 2p, one conditional subtraction after the wrap fix */
    uint64_t s = a + b;
    if (s < a) s += GL_EPS; /* wrapped past 2^64 */
    return canon(s);
}

static inline uint64_t gl_sub(uint64_t a, uint64_t b)
{
    return a >= b ? a - b : a + (GL_P - b);
}

/* 2^64 = 2^32 - 1 and 2^96 = -1 (mod p) */
static inline uint64_t gl_reduce(u128 x)
{
    uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
    uint64_t hh = hi >> 32, hl = hi & GL_EPS;
    uint64_t r = lo - hh;
    if (lo < hh) r -= GL_EPS;
    uint64_t m = (hl << 32) - hl;
    uint64_t s = r + m;
    if (s < r) s += GL_EPS;
    return canon(s);
}

static inline uint64_t gl_mul(uint64_t a, uint64_t b) { return gl_reduce((u128)a * b); }

static uint64_t gl_pow(uint64_t b, uint64_t e)
{
    uint64_t acc = 1;
    while (e) {
        if (e & 1) acc = gl_mul(acc, b);
        b = gl_mul(b, b);
        e >>= 1;
    }
    return acc;
}

static uint64_t gl_inv(uint64_t a) { return gl_pow(a, GL_P - 2); }

/* 2^k-th principal root of unity: the reference's W[k] table (goldilocks_base_field.cpp:11-44)
 * is W[32] = 0x64fdd1a46201e246 squared down, W[k] = W[k+1]^2. */
uint64_t orc_root_of_unity(unsigned k)
{
    uint64_t w = 0x64fdd1a46201e246ULL;
    for (unsigned i = 32; i > k; i--) w = gl_mul(w, w);
    return w;
}

uint64_t orc_mul(uint64_t a, uint64_t b) { return gl_mul(canon(a), canon(b)); }
uint64_t orc_add(uint64_t a, uint64_t b) { return gl_add(canon(a), canon(b)); }
uint64_t orc_sub(uint64_t a, uint64_t b) { return gl_sub(canon(a), canon(b)); }

/* ---------------------------------------------------------------- NTT ---- */

static unsigned log2u(uint64_t n)
{
    unsigned k = 0;
    while ((1ULL << k) < n) k++;
    return k;
}

static uint64_t bitrev(uint64_t x, unsigned bits)
{
    uint64_t r = 0;
    for (unsigned i = 0; i < bits; i++) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}

/* In-place radix-2 NTT of one contiguous vector: a[j] <- sum_i a[i] w^(ij),
 * w = W[log2 n] (or its inverse).  Textbook iterative Cooley-Tukey after a
 * bit-reversal permutation. */
static void ntt_vec(uint64_t *a, uint64_t n, int inverse)
{
    unsigned lg = log2u(n);
    for (uint64_t i = 0; i < n; i++) {
        uint64_t j = bitrev(i, lg);
        if (j > i) {
            uint64_t t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    for (unsigned s = 1; s <= lg; s++) {
        uint64_t m = 1ULL << s, half = m >> 1;
        uint64_t wm = orc_root_of_unity(s);
        if (inverse) wm = gl_inv(wm);
        uint64_t *tw = (uint64_t *)malloc(half * sizeof(uint64_t));
        tw[0] = 1;
        for (uint64_t j = 1; j < half; j++) tw[j] = gl_mul(tw[j - 1], wm);
        for (uint64_t k = 0; k < n; k += m)
            for (uint64_t j = 0; j < half; j++) {
                uint64_t t = gl_mul(tw[j], a[k + j + half]);
                uint64_t u = a[k + j];
                a[k + j] = gl_add(u, t);
                a[k + j + half] = gl_sub(u, t);
            }
        free(tw);
    }
    if (inverse) {
        uint64_t ninv = gl_inv(n % GL_P);
        for (uint64_t i = 0; i < n; i++) a[i] = gl_mul(a[i], ninv);
    }
}

/* forward (inverse=0) or inverse NTT of each column of a row-major n x ncols matrix */
void orc_ntt(uint64_t *dst, const uint64_t *src, uint64_t n, uint64_t ncols, int inverse)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (uint64_t c = 0; c < ncols; c++) {
        uint64_t *v = (uint64_t *)malloc(n * sizeof(uint64_t));
        for (uint64_t i = 0; i < n; i++) v[i] = canon(src[i * ncols + c]);
        ntt_vec(v, n, inverse);
        for (uint64_t i = 0; i < n; i++) dst[i * ncols + c] = v[i];
        free(v);
    }
}

/* LDE of one column: out[j] = p(7 * w_NExt^j), p the interpolant of in on <w_N>.
 * in: N words with stride in_stride; out: NExt words with stride out_stride. */
static void lde_col(uint64_t *out, uint64_t out_stride, const uint64_t *in, uint64_t in_stride, uint64_t N,
                    uint64_t NExt)
{
    uint64_t *v = (uint64_t *)calloc(NExt, sizeof(uint64_t));
    for (uint64_t i = 0; i < N; i++) v[i] = canon(in[i * in_stride]);
    ntt_vec(v, N, 1);
    uint64_t g = 1;
    for (uint64_t i = 0; i < N; i++) {
        v[i] = gl_mul(v[i], g);
        g = gl_mul(g, 7);
    }
    ntt_vec(v, NExt, 0);
    for (uint64_t j = 0; j < NExt; j++) out[j * out_stride] = v[j];
    free(v);
}

/* row-major in (N x ncols) -> row-major out (NExt x ncols) */
void orc_lde(uint64_t *out, const uint64_t *in, uint64_t N, uint64_t NExt, uint64_t ncols)
{
    if (N == 0 || ncols == 0) return;
#pragma omp parallel for schedule(dynamic, 1)
    for (uint64_t c = 0; c < ncols; c++) lde_col(out + c, ncols, in + c, ncols, N, NExt);
}

/* ---------------------------------------------------------- Poseidon2 ---- */

static const uint64_t *p2_c(unsigned w)
{
    return w == 4 ? P2_C4 : w == 8 ? P2_C8 : w == 12 ? P2_C12 : P2_C16;
}
static const uint64_t *p2_d(unsigned w)
{
    return w == 4 ? P2_D4 : w == 8 ? P2_D8 : w == 12 ? P2_D12 : P2_D16;
}

static inline uint64_t sbox(uint64_t x)
{
    uint64_t x2 = gl_mul(x, x);
    uint64_t x3 = gl_mul(x, x2);
    uint64_t x4 = gl_mul(x2, x2);
    return gl_mul(x3, x4);
}

/* the 4x4 block [[5,7,1,3],[4,6,1,1],[1,3,5,7],[1,1,4,6]] applied to x[0..4) */
static void m4(uint64_t *x)
{
    uint64_t a = x[0], b = x[1], c = x[2], d = x[3];
    uint64_t ab = gl_add(a, b), cd = gl_add(c, d);
    uint64_t bbcd = gl_add(gl_add(b, b), cd);    /* 2b + c + d */
    uint64_t ddab = gl_add(gl_add(d, d), ab);    /* a + b + 2d */
    uint64_t cd4 = gl_add(gl_add(cd, cd), gl_add(cd, cd));
    uint64_t ab4 = gl_add(gl_add(ab, ab), gl_add(ab, ab));
    uint64_t y3 = gl_add(cd4, ddab);             /* a + b + 4c + 6d */
    uint64_t y1 = gl_add(ab4, bbcd);             /* 4a + 6b + c + d */
    x[0] = gl_add(ddab, y1);                     /* 5a + 7b + c + 3d */
    x[1] = y1;
    x[2] = gl_add(bbcd, y3);                     /* a + 3b + 5c + 7d */
    x[3] = y3;
}

/* external layer: circ(2*M4, M4, ..., M4) = M4 per block, then add the block-column sums */
static void external_layer(uint64_t *x, unsigned w)
{
    for (unsigned i = 0; i < w; i += 4) m4(x + i);
    if (w > 4) {
        uint64_t s[4] = {0, 0, 0, 0};
        for (unsigned i = 0; i < w; i += 4)
            for (unsigned j = 0; j < 4; j++) s[j] = gl_add(s[j], x[i + j]);
        for (unsigned i = 0; i < w; i++) x[i] = gl_add(x[i], s[i & 3]);
    }
}

/* Poseidon2 permutation of a width-w state (w in 4, 8, 12, 16), in place */
void orc_permute(unsigned w, uint64_t *x)
{
    const uint64_t *C = p2_c(w), *D = p2_d(w);
    unsigned np = (w == 4) ? P2_NPARTIAL_4 : 22;
    for (unsigned i = 0; i < w; i++) x[i] = canon(x[i]);
    external_layer(x, w);
    for (unsigned r = 0; r < 4; r++) {
        for (unsigned i = 0; i < w; i++) x[i] = sbox(gl_add(x[i], C[r * w + i]));
        external_layer(x, w);
    }
    for (unsigned r = 0; r < np; r++) {
        x[0] = sbox(gl_add(x[0], C[4 * w + r]));
        uint64_t s = 0;
        for (unsigned i = 0; i < w; i++) s = gl_add(s, x[i]);
        for (unsigned i = 0; i < w; i++) x[i] = gl_add(gl_mul(x[i], D[i]), s);
    }
    for (unsigned r = 0; r < 4; r++) {
        for (unsigned i = 0; i < w; i++) x[i] = sbox(gl_add(x[i], C[4 * w + np + r * w + i]));
        external_layer(x, w);
    }
}

/* ---------------------------------------------------------- Poseidon1 ---- */

static int g_family = 2; /* 1 = Poseidon1, 2 = Poseidon2 */

void orc_set_hash_family(int family) { g_family = family == 1 ? 1 : 2; }
int orc_hash_family(void) { return g_family; }

/* out_i = sum_j mat[j][i] x_j (mat row-major w x w, applied transposed as mvp_ does) */
static void p1_mvp(uint64_t *x, const uint64_t *mat, unsigned w)
{
    uint64_t y[16];
    for (unsigned i = 0; i < w; i++) {
        uint64_t acc = 0;
        for (unsigned j = 0; j < w; j++) acc = gl_add(acc, gl_mul(mat[j * w + i], x[j]));
        y[i] = acc;
    }
    memcpy(x, y, w * sizeof(uint64_t));
}

/* Poseidon1 permutation of a width-w state (w in 8, 12, 16), in place: add C_0; 3 x (x^7, add
 * C_r, M); x^7, add C_4, P; 22 sparse partial rounds (x0^7 + c; x0' = <x, S_r[0..w)>;
 * x_i += x0 * S_r[w-1+i] for i >= 1); 3 x (x^7, add C, M); x^7, M. */
void orc_p1_permute(unsigned w, uint64_t *x)
{
    const uint64_t *C = w == 8 ? P1_C8 : w == 12 ? P1_C12 : P1_C16;
    const uint64_t *M = w == 8 ? P1_M8 : w == 12 ? P1_M12 : P1_M16;
    const uint64_t *P = w == 8 ? P1_P8 : w == 12 ? P1_P12 : P1_P16;
    const uint64_t *S = w == 8 ? P1_S8 : w == 12 ? P1_S12 : P1_S16;
    for (unsigned i = 0; i < w; i++) x[i] = gl_add(canon(x[i]), C[i]);
    for (unsigned r = 0; r < 3; r++) {
        for (unsigned i = 0; i < w; i++) x[i] = gl_add(sbox(x[i]), C[(r + 1) * w + i]);
        p1_mvp(x, M, w);
    }
    for (unsigned i = 0; i < w; i++) x[i] = gl_add(sbox(x[i]), C[4 * w + i]);
    p1_mvp(x, P, w);
    for (unsigned r = 0; r < P1_NPARTIAL; r++) {
        const uint64_t *Sr = S + (2 * w - 1) * r;
        const uint64_t x0 = gl_add(sbox(x[0]), C[5 * w + r]);
        x[0] = x0;
        uint64_t s0 = 0;
        for (unsigned i = 0; i < w; i++) s0 = gl_add(s0, gl_mul(x[i], Sr[i]));
        for (unsigned i = 1; i < w; i++) x[i] = gl_add(x[i], gl_mul(x0, Sr[w - 1 + i]));
        x[0] = s0;
    }
    for (unsigned r = 0; r < 3; r++) {
        for (unsigned i = 0; i < w; i++) x[i] = gl_add(sbox(x[i]), C[5 * w + P1_NPARTIAL + r * w + i]);
        p1_mvp(x, M, w);
    }
    for (unsigned i = 0; i < w; i++) x[i] = sbox(x[i]);
    p1_mvp(x, M, w);
}

/* the permutation of the selected family */
static void permute_fam(unsigned w, uint64_t *x)
{
    if (g_family == 1)
        orc_p1_permute(w, x);
    else
        orc_permute(w, x);
}

/* Sponge over `size` words with stride `stride`: rate w-4, capacity 4.  The capacity starts
 * at zero; each later block carries the previous output's first 4 words into it; a short
 * last block is zero-filled; no length padding; size 0 gives the zero digest. */
static void linear_hash_strided(unsigned w, uint64_t out[4], const uint64_t *in, uint64_t stride, uint64_t size)
{
    uint64_t st[16];
    unsigned rate = w - 4;
    memset(st, 0, sizeof(st));
    if (size == 0) {
        memset(out, 0, 4 * sizeof(uint64_t));
        return;
    }
    for (uint64_t done = 0; done < size;) {
        uint64_t n = size - done < rate ? size - done : rate;
        if (done > 0) memcpy(st + rate, st, 4 * sizeof(uint64_t));
        for (unsigned i = 0; i < rate; i++) st[i] = i < n ? canon(in[(done + i) * stride]) : 0;
        permute_fam(w, st);
        done += n;
    }
    memcpy(out, st, 4 * sizeof(uint64_t));
}

void orc_linear_hash(unsigned w, uint64_t out[4], const uint64_t *in, uint64_t size)
{
    linear_hash_strided(w, out, in, 1, size);
}

uint64_t orc_tree_num_elements(uint64_t nrows, uint64_t arity)
{
    uint64_t total = nrows, level = nrows;
    while (level > 1) {
        total += (arity - level % arity) % arity;
        level = (level + arity - 1) / arity;
        total += level;
    }
    return total * 4;
}

/* Fold digests level by level up to the root, in the reference buffer layout:
 * [level 0 digests | zero pad | level 1 | pad | ... | root].  Parent i of a level hashes the
 * arity*4 = w contiguous words of its children with one permutation and keeps words 0..3. */
static void build_levels_w(uint64_t *tree, uint64_t nleaves, uint64_t arity, unsigned w)
{
    uint64_t pending = nleaves, base = 0;
    while (pending > 1) {
        uint64_t pad = (arity - pending % arity) % arity;
        memset(tree + base + pending * 4, 0, pad * 4 * sizeof(uint64_t));
        uint64_t parents = (pending + arity - 1) / arity;
        uint64_t *dst = tree + base + (pending + pad) * 4;
#pragma omp parallel for schedule(static)
        for (uint64_t i = 0; i < parents; i++) {
            uint64_t st[16];
            memset(st, 0, sizeof(st));
            memcpy(st, tree + base + i * 4 * arity, 4 * arity * sizeof(uint64_t));
            permute_fam(w, st);
            memcpy(dst + i * 4, st, 4 * sizeof(uint64_t));
        }
        base += (pending + pad) * 4;
        pending = parents;
    }
}

static void build_levels(uint64_t *tree, uint64_t nleaves, uint64_t arity)
{
    build_levels_w(tree, nleaves, arity, (unsigned)(4 * arity));
}

/* Merkle tree of an nrows x ncols matrix given by (row_stride, col_stride); W = 4 * arity */
static int merkletree_strided(uint64_t *tree, const uint64_t *in, uint64_t row_stride, uint64_t col_stride,
                              uint64_t ncols, uint64_t nrows, uint64_t arity)
{
    if (arity < 2 || arity > 4) return -1;
    if (nrows == 0) return 0;
    unsigned w = (unsigned)(4 * arity);
#pragma omp parallel for schedule(static)
    for (uint64_t r = 0; r < nrows; r++) linear_hash_strided(w, tree + r * 4, in + r * row_stride, col_stride, ncols);
    build_levels(tree, nrows, arity);
    return 0;
}

/* row-major input (reference CPU layout) */
int orc_merkletree(uint64_t *tree, const uint64_t *in, uint64_t ncols, uint64_t nrows, uint64_t arity)
{
    return merkletree_strided(tree, in, ncols, 1, ncols, nrows, arity);
}

/* column-major input (col * nrows + row, the device layout) */
int orc_merkletree_colmajor(uint64_t *tree, const uint64_t *in, uint64_t ncols, uint64_t nrows, uint64_t arity)
{
    return merkletree_strided(tree, in, 1, nrows, ncols, nrows, arity);
}

/* row-major input, sponge and node width w with 4 * arity <= w (PoseidonGoldilocks<W>::merkletree
 * pads each node's arity*4 child words with zeros up to W) */
int orc_merkletree_w(unsigned w, uint64_t *tree, const uint64_t *in, uint64_t ncols, uint64_t nrows, uint64_t arity)
{
    if (arity < 2 || 4 * arity > w) return -1;
    if (nrows == 0) return 0;
#pragma omp parallel for schedule(static)
    for (uint64_t r = 0; r < nrows; r++) linear_hash_strided(w, tree + r * 4, in + r * ncols, 1, ncols);
    build_levels_w(tree, nrows, arity, w);
    return 0;
}

int orc_merkletree_reduce(unsigned w, uint64_t root[4], const uint64_t *digests, uint64_t n, uint64_t arity)
{
    if (4 * arity != w) return -1;
    uint64_t total = orc_tree_num_elements(n, arity);
    uint64_t *t = (uint64_t *)calloc(total, sizeof(uint64_t));
    for (uint64_t i = 0; i < 4 * n; i++) t[i] = canon(digests[i]);
    build_levels(t, n, arity);
    memcpy(root, t + total - 4, 4 * sizeof(uint64_t));
    free(t);
    return 0;
}

/* LDE + tree of a row-major trace (write_custom_commit_cpu, api/starks_api.cpp:633-657).
 * lde: NExt x ncols row-major (may be NULL); tree: orc_tree_num_elements words (may be NULL). */
int orc_commit(uint64_t root[4], uint64_t *lde, uint64_t *tree, const uint64_t *trace, uint64_t nBits,
               uint64_t nBitsExt, uint64_t ncols, uint64_t arity)
{
    uint64_t N = 1ULL << nBits, NExt = 1ULL << nBitsExt;
    if (arity < 2 || arity > 4 || nBitsExt < nBits) return -1;
    uint64_t *l = lde ? lde : (uint64_t *)malloc(NExt * ncols * sizeof(uint64_t));
    uint64_t total = orc_tree_num_elements(NExt, arity);
    uint64_t *t = tree ? tree : (uint64_t *)malloc(total * sizeof(uint64_t));
    orc_lde(l, trace, N, NExt, ncols);
    int rc = orc_merkletree(t, l, ncols, NExt, arity);
    memcpy(root, t + total - 4, 4 * sizeof(uint64_t));
    if (!lde) free(l);
    if (!tree) free(t);
    return rc;
}

/* ------------------------------------------------------ query openings ---- */

static uint64_t ipow_u(uint64_t b, uint64_t e)
{
    uint64_t r = 1;
    while (e--) r *= b;
    return r;
}

/* MerkleTreeGL::getGroupProof (merkleTreeGL.cpp:145-175): the row's ncols words, then per level
 * the (arity-1) sibling digests of the path node in child order, until the root or until a level
 * has <= arity^llv nodes.  lde is row-major nrows x ncols; returns the number of words written. */
uint64_t orc_group_proof(uint64_t *out, const uint64_t *lde, uint64_t nrows, uint64_t ncols, const uint64_t *tree,
                         uint64_t arity, uint64_t llv, uint64_t row)
{
    uint64_t w = 0;
    for (uint64_t c = 0; c < ncols; c++) out[w++] = canon(lde[row * ncols + c]);
    uint64_t idx = row, offset = 0, n = nrows;
    const uint64_t stop = llv ? ipow_u(arity, llv) : 1;
    while (llv ? (n > stop) : (n > 1)) {
        const uint64_t cur = idx % arity, si = idx - cur;
        for (uint64_t i = 0; i < arity; i++) {
            if (i == cur) continue;
            for (int j = 0; j < 4; j++) out[w++] = tree[(offset + si + i) * 4 + j];
        }
        const uint64_t next = (n + arity - 1) / arity;
        offset += next * arity;
        idx /= arity;
        n = next;
    }
    return w;
}

/* Recompute the root (llv = 0) from an opening: leaf = linear hash of the row, then one
 * permutation per level over the arity children with the path node at its position
 * (MerkleTreeGL::verifyGroupProof / calculateRootFromProof, merkleTreeGL.cpp:177-296). */
void orc_root_from_proof(uint64_t root[4], const uint64_t *proof, uint64_t ncols, uint64_t nrows, uint64_t arity,
                         uint64_t row)
{
    unsigned w = (unsigned)(4 * arity);
    uint64_t h[4];
    linear_hash_strided(w, h, proof, 1, ncols);
    const uint64_t *sib = proof + ncols;
    uint64_t idx = row, n = nrows;
    while (n > 1) {
        const uint64_t cur = idx % arity;
        uint64_t st[16];
        unsigned p = 0;
        for (uint64_t i = 0; i < arity; i++) {
            const uint64_t *src = (i == cur) ? h : sib + 4 * (p++);
            memcpy(st + 4 * i, src, 32);
        }
        sib += 4 * (arity - 1);
        permute_fam(w, st);
        memcpy(h, st, 32);
        idx /= arity;
        n = (n + arity - 1) / arity;
    }
    memcpy(root, h, 32);
}

/* ------------------------------------------------------------ Q-stage commit ---- */

/* Starks::computeQ (starks.hpp:186-239): q is row-major NExt x qDim (evaluations); each limb
 * column is inverse-transformed over NExt; coefficient p*N + i of limb k, times
 * S[p] = (7^-1)^(N*p), becomes row i of cmQ column p*qDim + k (rows N..NExt-1 zero); each cmQ
 * column is forward-transformed over NExt; then the Merkle tree of cmQ (row-major NExt x
 * qDeg*qDim).  cmq and tree may be NULL. */
int orc_commit_q(uint64_t root[4], uint64_t *cmq, uint64_t *tree, const uint64_t *q, uint64_t nBits, uint64_t nBitsExt,
                 uint64_t qDeg, uint64_t qDim, uint64_t arity)
{
    const uint64_t N = 1ULL << nBits, NExt = 1ULL << nBitsExt, ncols = qDeg * qDim;
    if (nBitsExt < nBits || qDeg * N > NExt || arity < 2 || arity > 4) return -1;
    uint64_t *coef = (uint64_t *)malloc(NExt * qDim * sizeof(uint64_t));
    orc_ntt(coef, q, NExt, qDim, 1);
    uint64_t *cm = cmq ? cmq : (uint64_t *)malloc(NExt * ncols * sizeof(uint64_t));
    memset(cm, 0, NExt * ncols * sizeof(uint64_t));
    const uint64_t shift_in = gl_pow(gl_inv(7), N);
    uint64_t S = 1;
    for (uint64_t p = 0; p < qDeg; p++) {
        for (uint64_t i = 0; i < N; i++)
            for (uint64_t k = 0; k < qDim; k++) cm[i * ncols + p * qDim + k] = gl_mul(coef[(p * N + i) * qDim + k], S);
        S = gl_mul(S, shift_in);
    }
    free(coef);
    orc_ntt(cm, cm, NExt, ncols, 0);
    const uint64_t total = orc_tree_num_elements(NExt, arity);
    uint64_t *t = tree ? tree : (uint64_t *)malloc(total * sizeof(uint64_t));
    int rc = orc_merkletree(t, cm, ncols, NExt, arity);
    memcpy(root, t + total - 4, 4 * sizeof(uint64_t));
    if (!cmq) free(cm);
    if (!tree) free(t);
    return rc;
}
