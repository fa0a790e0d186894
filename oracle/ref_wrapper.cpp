// C entry points over the reference's own CPU implementation of the commit path.
//
// Test infrastructure: compiled by oracle/Makefile together with the unmodified
// reference sources goldilocks_base_field.cpp, ntt_goldilocks.cpp, poseidon2_goldilocks.cpp and
// poseidon_goldilocks.cpp into oracle/_ref/libpil2ref_*.so.  Used by the tests
// as a second, independent checker of the CUDA path and by bench.py as the
// timed reference CPU baseline.  Every function mirrors one reference call:
//   ref_lde          -> NTT_Goldilocks::LDE                 (ntt_goldilocks.cpp:369-404)
//   ref_ntt          -> NTT_Goldilocks::NTT / INTT          (ntt_goldilocks.cpp:211-260)
//   ref_merkletree   -> Poseidon2Goldilocks<W>::merkletree  (poseidon2_goldilocks.hpp:337-369),
//                       W = 4*arity as MerkleTreeGL::merkelize picks it (merkleTreeGL.cpp:316-336)
//   ref_commit       -> write_custom_commit_cpu             (api/starks_api.cpp:633-657)
//   ref_p1_*         -> PoseidonGoldilocks<W> (Poseidon1)   (poseidon_goldilocks.hpp:30-76), the
//                       hash family 1 branch of MerkleTreeGL::merkelize (merkleTreeGL.cpp:300-318)
#include <cstdint>
#include <cstring>
#include <vector>

#include "goldilocks_base_field.hpp"
#include "goldilocks_tooling.hpp"
#include "ntt_goldilocks.hpp"
#include "poseidon2_goldilocks.hpp"
#include "poseidon_goldilocks.hpp"

using GE = Goldilocks::Element;

extern "C" {

int ref_has_avx512(void)
{
#ifdef __AVX512__
    return 1;
#else
    return 0;
#endif
}

void ref_set_threads(int n) { omp_set_num_threads(n); }

int ref_max_threads(void) { return omp_get_max_threads(); }

uint64_t ref_tree_num_elements(uint64_t nrows, uint64_t arity) { return getTreeNumElements(nrows, (uint32_t)arity); }

// Row-major LDE: out is NExt x ncols, in is N x ncols. buffer may be NULL.
void ref_lde(uint64_t *out, const uint64_t *in, uint64_t N, uint64_t NExt, uint64_t ncols, uint64_t *buffer,
             uint64_t nblock)
{
    NTT_Goldilocks ntt(N);
    ntt.LDE((GE *)out, (GE *)in, NExt, N, ncols, (GE *)buffer, NUM_PHASES, nblock == 0 ? 1 : nblock);
}

void ref_ntt(uint64_t *dst, const uint64_t *src, uint64_t size, uint64_t ncols, int inverse)
{
    NTT_Goldilocks ntt(size);
    if (inverse)
        ntt.INTT((GE *)dst, (GE *)src, size, ncols);
    else
        ntt.NTT((GE *)dst, (GE *)src, size, ncols);
}

static int width_for_arity(uint64_t arity) { return arity == 2 ? 8 : arity == 3 ? 12 : arity == 4 ? 16 : 0; }

// tree must hold ref_tree_num_elements(nrows, arity) words; input row-major nrows x ncols.
int ref_merkletree(uint64_t *tree, const uint64_t *input, uint64_t ncols, uint64_t nrows, uint64_t arity)
{
    switch (width_for_arity(arity)) {
    case 8: Poseidon2Goldilocks<8>::merkletree((GE *)tree, (GE *)input, ncols, nrows, arity); return 0;
    case 12: Poseidon2Goldilocks<12>::merkletree((GE *)tree, (GE *)input, ncols, nrows, arity); return 0;
    case 16: Poseidon2Goldilocks<16>::merkletree((GE *)tree, (GE *)input, ncols, nrows, arity); return 0;
    default: return -1;
    }
}

int ref_permute(uint64_t width, uint64_t *out, const uint64_t *in)
{
    switch (width) {
    case 4: Poseidon2Goldilocks<4>::permute(*(GE(*)[4])out, *(const GE(*)[4])in, Poseidon2Mode::Scalar); return 0;
    case 8: Poseidon2Goldilocks<8>::permute(*(GE(*)[8])out, *(const GE(*)[8])in, Poseidon2Mode::Scalar); return 0;
    case 12: Poseidon2Goldilocks<12>::permute(*(GE(*)[12])out, *(const GE(*)[12])in, Poseidon2Mode::Scalar); return 0;
    case 16: Poseidon2Goldilocks<16>::permute(*(GE(*)[16])out, *(const GE(*)[16])in, Poseidon2Mode::Scalar); return 0;
    default: return -1;
    }
}

int ref_linear_hash(uint64_t width, uint64_t *out, const uint64_t *in, uint64_t size)
{
    std::vector<GE> tmp(size + 1);
    if (size) std::memcpy(tmp.data(), in, size * 8);
    switch (width) {
    case 8: Poseidon2Goldilocks<8>::linearHash((GE *)out, tmp.data(), size, Poseidon2Mode::Scalar); return 0;
    case 12: Poseidon2Goldilocks<12>::linearHash((GE *)out, tmp.data(), size, Poseidon2Mode::Scalar); return 0;
    case 16: Poseidon2Goldilocks<16>::linearHash((GE *)out, tmp.data(), size, Poseidon2Mode::Scalar); return 0;
    default: return -1;
    }
}

int ref_merkletree_reduce(uint64_t width, uint64_t *root, const uint64_t *digests, uint64_t n, uint64_t arity)
{
    std::vector<GE> tmp(4 * n + 4);
    std::memcpy(tmp.data(), digests, 4 * n * 8);
    switch (width) {
    case 8: Poseidon2Goldilocks<8>::merkletreeReduce((GE *)root, tmp.data(), n, arity); return 0;
    case 12: Poseidon2Goldilocks<12>::merkletreeReduce((GE *)root, tmp.data(), n, arity); return 0;
    case 16: Poseidon2Goldilocks<16>::merkletreeReduce((GE *)root, tmp.data(), n, arity); return 0;
    default: return -1;
    }
}

// LDE + Merkle tree of a row-major trace, as write_custom_commit_cpu does.
// lde (NExt*ncols words, row-major) and tree (ref_tree_num_elements words) are caller-owned.
int ref_commit(uint64_t *root, uint64_t *lde, uint64_t *tree, const uint64_t *trace, uint64_t nBits,
               uint64_t nBitsExt, uint64_t ncols, uint64_t arity, uint64_t nblock)
{
    uint64_t N = 1ULL << nBits, NExt = 1ULL << nBitsExt;
    ref_lde(lde, trace, N, NExt, ncols, nullptr, nblock);
    int rc = ref_merkletree(tree, lde, ncols, NExt, arity);
    if (rc) return rc;
    uint64_t n = getTreeNumElements(NExt, (uint32_t)arity);
    for (int i = 0; i < 4; i++) root[i] = Goldilocks::toU64(((GE *)tree)[n - 4 + i]);
    return 0;
}

// Starks::computeQ (pil2-stark/src/starkpil/starks.hpp:186-239) on the reference's NTT and field
// code: q (row-major NExt x qDim evaluations) -> INTT over NExt -> chunk p of N coefficients times
// S[p] = (shift^-1)^(N*p) into cmQ[(i*qDeg + p)*qDim + k] -> zero rows N..NExt -> NTT over NExt ->
// Poseidon2 tree.  The reference multiplies each chunk as a cubic-extension element by the base
// scalar S[p] (Goldilocks3::mul), i.e. limb by limb, which is what the loop below does for any qDim.
// cmq: NExt x (qDeg*qDim) row-major, tree: ref_tree_num_elements(NExt, arity) words.
int ref_commit_q(uint64_t *root, uint64_t *cmq, uint64_t *tree, const uint64_t *q, uint64_t nBits, uint64_t nBitsExt,
                 uint64_t qDeg, uint64_t qDim, uint64_t arity)
{
    const uint64_t N = 1ULL << nBits, NExt = 1ULL << nBitsExt, ncols = qDeg * qDim;
    if (nBitsExt < nBits || qDeg == 0 || qDim == 0 || qDeg * N > NExt) return -1;
    std::vector<GE> coef(NExt * qDim);
    std::memcpy(coef.data(), q, NExt * qDim * 8);
    NTT_Goldilocks nttExtended(NExt);
    nttExtended.INTT(coef.data(), coef.data(), NExt, qDim);
    std::vector<GE> S(qDeg);
    const GE shiftIn = Goldilocks::exp(Goldilocks::inv(Goldilocks::shift()), N);
    S[0] = Goldilocks::one();
    for (uint64_t p = 1; p < qDeg; p++) S[p] = Goldilocks::mul(S[p - 1], shiftIn);
    GE *cm = (GE *)cmq;
#pragma omp parallel for collapse(2)
    for (uint64_t p = 0; p < qDeg; p++)
        for (uint64_t i = 0; i < N; i++)
            for (uint64_t k = 0; k < qDim; k++)
                cm[(i * qDeg + p) * qDim + k] = Goldilocks::mul(coef[(p * N + i) * qDim + k], S[p]);
#pragma omp parallel for
    for (uint64_t i = N * ncols; i < NExt * ncols; i++) cm[i] = Goldilocks::zero();
    nttExtended.NTT(cm, cm, NExt, ncols);
    int rc = ref_merkletree(tree, cmq, ncols, NExt, arity);
    if (rc) return rc;
    const uint64_t n = getTreeNumElements(NExt, (uint32_t)arity);
    for (int i = 0; i < 4; i++) root[i] = Goldilocks::toU64(((GE *)tree)[n - 4 + i]);
    return 0;
}

// Seeded test data: element i of stream `seed` is the first splitmix64 output below p keyed by
// (seed, i, j), j = 0, 1, ...  The same rule as the product's b200_fill_random_host/_device, so
// a device-filled trace and a trace filled here are identical without either side loading the
// other's library.
static inline uint64_t fill_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

void ref_fill_random(uint64_t *buf, uint64_t n, uint64_t seed)
{
    const uint64_t key0 = fill_mix64(seed * 0x9e3779b97f4a7c15ULL + 0x632be59bd9b4e019ULL);
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < n; i++) {
        const uint64_t key = key0 ^ (i * 0x9e3779b97f4a7c15ULL);
        uint64_t v;
        for (uint64_t j = 0;; j++) {
            v = fill_mix64(key + j * 0xd1b54a32d192ed03ULL);
            if (v < 0xFFFFFFFF00000001ULL) break;
        }
        buf[i] = v;
    }
}

// Canonicalise a buffer in place (x mod p), the form every comparison uses.
void ref_canonicalize(uint64_t *buf, uint64_t n)
{
#pragma omp parallel for
    for (uint64_t i = 0; i < n; i++) buf[i] = Goldilocks::toU64(((GE *)buf)[i]);
}

// ---- Poseidon1 (hash family 1) ----
int ref_p1_permute(uint64_t width, uint64_t *out, const uint64_t *in)
{
    switch (width) {
    case 8: PoseidonGoldilocks<8>::permute(*(GE(*)[8])out, *(const GE(*)[8])in, PoseidonMode::Scalar); return 0;
    case 12: PoseidonGoldilocks<12>::permute(*(GE(*)[12])out, *(const GE(*)[12])in, PoseidonMode::Scalar); return 0;
    case 16: PoseidonGoldilocks<16>::permute(*(GE(*)[16])out, *(const GE(*)[16])in, PoseidonMode::Scalar); return 0;
    default: return -1;
    }
}

int ref_p1_linear_hash(uint64_t width, uint64_t *out, const uint64_t *in, uint64_t size)
{
    std::vector<GE> tmp(size + 1);
    if (size) std::memcpy(tmp.data(), in, size * 8);
    switch (width) {
    case 8: PoseidonGoldilocks<8>::linearHash((GE *)out, tmp.data(), size, PoseidonMode::Scalar); return 0;
    case 12: PoseidonGoldilocks<12>::linearHash((GE *)out, tmp.data(), size, PoseidonMode::Scalar); return 0;
    case 16: PoseidonGoldilocks<16>::linearHash((GE *)out, tmp.data(), size, PoseidonMode::Scalar); return 0;
    default: return -1;
    }
}

// width 0: W = 4*arity (MerkleTreeGL's choice); otherwise the given W with 4*arity <= W
int ref_p1_merkletree(uint64_t width, uint64_t *tree, const uint64_t *input, uint64_t ncols, uint64_t nrows,
                      uint64_t arity)
{
    const uint64_t w = width ? width : (uint64_t)width_for_arity(arity);
    if (4 * arity > w) return -1;
    switch (w) {
    case 8: PoseidonGoldilocks<8>::merkletree((GE *)tree, (GE *)input, ncols, nrows, arity); return 0;
    case 12: PoseidonGoldilocks<12>::merkletree((GE *)tree, (GE *)input, ncols, nrows, arity); return 0;
    case 16: PoseidonGoldilocks<16>::merkletree((GE *)tree, (GE *)input, ncols, nrows, arity); return 0;
    default: return -1;
    }
}

}  // extern "C"
