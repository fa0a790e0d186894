// Streaming slot commit of a bit-packed witness (the reference's streamCommitPacked,
// goldilocks/src/stream_commit.cu, reached through commit_witness_streaming,
// api/starks_api.cu:2290-2348).
//
// Instead of materialising the NExt x nCols LDE and hashing rows, the columns are processed in
// chunks of RATE = W - 4: each chunk is unpacked (column-major, N rows), extended in place by the
// LDE, and absorbed into the row sponge: rate words = the chunk's extended values (zero-filled
// past the last column), capacity = the previous block's first four output words (zero for the
// first chunk).  That is the linear hash of the whole row, block by block, so after the last
// chunk the four carried words are the leaf digests; the tree levels follow.  Working set per
// slot: the packed witness, the tree (whose level 0 holds the carried words), one chunk's LDE
// (RATE x NExt) and one chunk's unpacked columns (RATE x N).
#pragma once
#include "merkle.cuh"
#include "ntt.cuh"
#include "unpack.cuh"

namespace stream {

constexpr uint64_t MAX_COLS = 64;  // widest witness a slot accepts (the reference's SC_MAX_COLS)

struct Layout {
    uint64_t widths, offsets, packed, tree, chunk, scratch, total;  // word offsets / size
};

// rate = W - 4 of the W = 16 sponge the slot commit uses (arity 4)
constexpr uint32_t RATE = 12;

inline Layout layout(uint64_t nBits, uint64_t nBitsExt, uint64_t wordsPerRow)
{
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    Layout l;
    auto up = [](uint64_t x) { return (x + 31) & ~31ull; };  // 256-byte aligned regions
    l.widths = 0;
    l.offsets = MAX_COLS;
    l.packed = 2 * MAX_COLS;
    l.tree = up(l.packed + N * wordsPerRow);
    l.chunk = up(l.tree + merkle::tree_num_elements(NExt, 4));
    l.scratch = up(l.chunk + RATE * NExt);
    l.total = up(l.scratch + RATE * N);
    return l;
}

// columns [c0, c0 + cc) of the packed rows into cc column-major columns of dst (stride nrows);
// offsets[c] = bit offset of column c within a row (prefix sums of the widths)
__global__ void __launch_bounds__(256) unpack_range_kernel(uint64_t *__restrict__ dst, const uint64_t *__restrict__ src,
                                                           const uint64_t *__restrict__ widths,
                                                           const uint64_t *__restrict__ offsets, uint64_t nrows,
                                                           uint64_t words_per_row, uint32_t c0, uint32_t cc)
{
    const uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nrows) return;
    const uint64_t *w = src + row * words_per_row;
    for (uint32_t i = 0; i < cc; i++) {
        const uint64_t nb = widths[c0 + i], off = offsets[c0 + i];
        const uint64_t wi = off >> 6, sh = off & 63;
        uint64_t val = __ldg(w + wi) >> sh;
        if (sh + nb > 64) val |= __ldg(w + wi + 1) << (64 - sh);
        if (nb < 64) val &= (1ull << nb) - 1;
        dst[(uint64_t)i * nrows + row] = val;
    }
}

// Absorb one chunk of cc <= RATE extended columns (column-major, stride nrows) into the carried
// words `carry` (row-major, 4 per row = tree level 0).
template <int FAM>
__global__ void __launch_bounds__(merkle::TPB, merkle::Family<FAM>::MIN_CTAS) absorb_kernel(uint64_t *__restrict__ carry,
                                                             const uint64_t *__restrict__ chunk, uint32_t cc,
                                                             int first, uint64_t nrows)
{
    constexpr int W = 16;
    constexpr int TPB = merkle::TPB;
    __shared__ uint64_t sm[merkle::Family<FAM>::SMEM_AREAS * W * TPB];
    const uint64_t row = (uint64_t)blockIdx.x * TPB + threadIdx.x;
    if (row >= nrows) return;
    uint64_t *st = sm + threadIdx.x;
#pragma unroll
    for (uint32_t i = 0; i < RATE; i++) st[i * TPB] = i < cc ? __ldg(chunk + (uint64_t)i * nrows + row) : 0ull;
#pragma unroll
    for (int i = 0; i < 4; i++) st[(RATE + i) * TPB] = first ? 0ull : carry[row * 4 + i];
    merkle::permute_fam<W, FAM>(st);
#pragma unroll
    for (int i = 0; i < 4; i++) carry[row * 4 + i] = gl::canon(st[i * TPB]);
}

// Indexed witness: the instruction table on the device and the row header width; the slot's
// width region then holds width | source << 32 per column (unpack::bitfield_unpack_kernel).
struct Indexed {
    const uint64_t *table;
    uint64_t num_entries, words_per_entry, index_bits;
};

// The whole slot commit on `s` (device work only; the caller copies the packed rows to
// slot + layout.packed and the widths/offsets to their regions first).  Leaves the tree at
// slot + layout.tree.
template <int FAM>
inline cudaError_t run(uint64_t *slot, const Layout &l, uint64_t nBits, uint64_t nBitsExt, uint64_t nCols,
                       uint64_t wordsPerRow, cudaStream_t s, const Indexed *ix = nullptr)
{
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    uint64_t *tree = slot + l.tree, *chunk = slot + l.chunk, *scr = slot + l.scratch;
    cudaError_t e;
    for (uint64_t c0 = 0; c0 < nCols; c0 += RATE) {
        const uint32_t cc = (uint32_t)((nCols - c0) < RATE ? (nCols - c0) : RATE);
        if (ix) {
            e = unpack::launch(scr, slot + l.packed, ix->table, N, wordsPerRow, ix->words_per_entry, ix->num_entries,
                               (uint32_t)ix->index_bits, unpack::InfoDev{slot + l.widths}, (uint32_t)c0, cc, s);
            if (e != cudaSuccess) return e;
        } else {
            unpack_range_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(scr, slot + l.packed, slot + l.widths,
                                                                           slot + l.offsets, N, wordsPerRow,
                                                                           (uint32_t)c0, cc);
        }
        prof::count();
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if ((e = ntt::lde(chunk, scr, false, (uint32_t)nBits, (uint32_t)nBitsExt, cc, scr, s)) != cudaSuccess) return e;
        absorb_kernel<FAM><<<(unsigned)((NExt + merkle::TPB - 1) / merkle::TPB), merkle::TPB, 0, s>>>(
            tree, chunk, cc, c0 == 0, NExt);
        prof::count();
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return merkle::build_levels<16, FAM>(tree, NExt, s);
}

}  // namespace stream
