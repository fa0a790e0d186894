// Bit-packed (and indexed) witness -> column-major trace, in place of the transpose in front of
// the LDE.
//
// Packed layout (the reference's PackedInfo / unpack kernel, starks_gpu.cu:49-103): every row
// is `words_per_row` u64 words; column c occupies the next col_bits[c] bits, least
// significant first, and may straddle a word boundary.  The host trace shrinks from
// 64*nCols to sum(col_bits) bits per row, which is what crosses PCIe.  One thread per row walks
// its words and writes element (row, c) to dst[c*N + row] (consecutive threads, consecutive
// rows: coalesced stores).
#pragma once
#include <stdint.h>

namespace unpack {

// Column descriptions passed by value in the kernel parameters (no device allocation or copy
// per call): one byte per column, width 1..64 in bits 0-6, table source (indexed witness) in
// bit 7.  12 KB, inside the 32 KB kernel-parameter limit.
constexpr uint32_t COLS_MAX = 12288;
struct ColBytes {
    uint8_t v[COLS_MAX];
};

__global__ void __launch_bounds__(256) unpack_kernel(uint64_t *__restrict__ dst, const uint64_t *__restrict__ src,
                                                     uint64_t nrows, uint64_t ncols, uint64_t words_per_row,
                                                     const __grid_constant__ ColBytes cols)
{
    const uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nrows) return;
    const uint64_t *w = src + row * words_per_row;
    uint64_t word = words_per_row ? __ldg(w) : 0, idx = 0, off = 0;
    for (uint64_t c = 0; c < ncols; c++) {
        const uint32_t nb = cols.v[c] & 127u;
        uint64_t val;
        const uint64_t left = 64 - off;
        if (nb <= left) {
            const uint64_t mask = nb == 64 ? ~0ull : ((1ull << nb) - 1);
            val = (word >> off) & mask;
            off += nb;
            if (off == 64 && idx + 1 < words_per_row) {
                word = __ldg(w + ++idx);
                off = 0;
            }
        } else {
            const uint64_t low = word >> off;
            word = __ldg(w + ++idx);
            const uint64_t high = word & ((1ull << (nb - left)) - 1);
            val = (high << left) | low;
            off = nb - left;
        }
        dst[c * nrows + row] = val;
    }
}

// Bit cursor over a packed stream of `words` u64 words: take the next nb (1..64) bits, least
// significant first, crossing into the next word when needed.  The same walk as unpack_kernel.
struct Cursor {
    const uint64_t *base;
    uint64_t words, word, idx, off;
    __device__ __forceinline__ void start(const uint64_t *b, uint64_t n)
    {
        base = b;
        words = n;
        word = n ? __ldg(b) : 0;
        idx = 0;
        off = 0;
    }
    template <bool EXTRACT>
    __device__ __forceinline__ uint64_t take(uint64_t nb)
    {
        uint64_t val = 0;
        const uint64_t left = 64 - off;
        if (nb <= left) {
            if (EXTRACT) val = (word >> off) & (nb == 64 ? ~0ull : ((1ull << nb) - 1));
            off += nb;
            if (off == 64 && idx + 1 < words) {
                word = __ldg(base + ++idx);
                off = 0;
            }
        } else {
            const uint64_t low = word >> off;
            word = __ldg(base + ++idx);
            if (EXTRACT) val = ((word & ((1ull << (nb - left)) - 1)) << left) | low;
            off = nb - left;
        }
        return val;
    }
};

// Column info of the indexed kernels: width | source << 32, from device memory (the streaming
// slot's table) or from the kernel parameters.
struct InfoDev {
    const uint64_t *p;
};
__device__ __forceinline__ uint64_t col_info(const InfoDev &t, uint32_t c) { return __ldg(t.p + c); }
__device__ __forceinline__ uint64_t col_info(const ColBytes &t, uint32_t c)
{
    const uint32_t b = t.v[c];
    return (uint64_t)(b & 127u) | ((uint64_t)(b >> 7) << 32);
}

// Indexed witness (the reference's unpack_indexed, starks_gpu.cu:125-185): a row is a leading
// instruction index (index_bits wide) followed by the runtime columns; the columns flagged as
// table columns are read instead from entry `index` of a shared instruction table
// (words_per_entry words per entry, its own bit cursor).  An index past the table selects entry
// 0, as the reference does.  Columns [c0, c0 + cc) are written (column-major, stride nrows);
// earlier columns only advance the cursors.
template <class Info>
__device__ __forceinline__ void unpack_indexed_body(uint64_t *__restrict__ dst, const uint64_t *__restrict__ rows,
                                                    const uint64_t *__restrict__ table, uint64_t nrows,
                                                    uint64_t words_per_row, uint64_t words_per_entry,
                                                    uint64_t num_entries, uint64_t index_bits, const Info &info,
                                                    uint32_t c0, uint32_t cc)
{
    const uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nrows) return;
    Cursor r, t;
    r.start(rows + row * words_per_row, words_per_row);
    uint64_t index = index_bits ? r.take<true>(index_bits) : 0;
    if (index >= num_entries) index = 0;
    t.start(table + index * words_per_entry, words_per_entry);
    for (uint32_t c = 0; c < c0 + cc; c++) {
        const uint64_t ci = col_info(info, c), nb = ci & 0xffffffffull;
        if (ci >> 32) {
            if (c < c0)
                t.take<false>(nb);
            else
                dst[(uint64_t)(c - c0) * nrows + row] = t.take<true>(nb);
        } else {
            if (c < c0)
                r.take<false>(nb);
            else
                dst[(uint64_t)(c - c0) * nrows + row] = r.take<true>(nb);
        }
    }
}

// col_info in device memory (width | source << 32 per column)
__global__ void __launch_bounds__(256) unpack_indexed_kernel(uint64_t *__restrict__ dst,
                                                             const uint64_t *__restrict__ rows,
                                                             const uint64_t *__restrict__ table, uint64_t nrows,
                                                             uint64_t words_per_row, uint64_t words_per_entry,
                                                             uint64_t num_entries, uint64_t index_bits,
                                                             const uint64_t *__restrict__ col_info, uint32_t c0,
                                                             uint32_t cc)
{
    unpack_indexed_body(dst, rows, table, nrows, words_per_row, words_per_entry, num_entries, index_bits,
                        InfoDev{col_info}, c0, cc);
}

// column bytes in the kernel parameters
__global__ void __launch_bounds__(256) unpack_indexed_param_kernel(uint64_t *__restrict__ dst,
                                                                   const uint64_t *__restrict__ rows,
                                                                   const uint64_t *__restrict__ table, uint64_t nrows,
                                                                   uint64_t words_per_row, uint64_t words_per_entry,
                                                                   uint64_t num_entries, uint64_t index_bits,
                                                                   const __grid_constant__ ColBytes cols, uint32_t c0,
                                                                   uint32_t cc)
{
    unpack_indexed_body(dst, rows, table, nrows, words_per_row, words_per_entry, num_entries, index_bits, cols, c0,
                        cc);
}

// bits of a packed row (host check of words_per_row)
inline uint64_t packed_bits(const uint32_t *col_bits, uint64_t ncols)
{
    uint64_t s = 0;
    for (uint64_t c = 0; c < ncols; c++) s += col_bits[c];
    return s;
}

}  // namespace unpack
