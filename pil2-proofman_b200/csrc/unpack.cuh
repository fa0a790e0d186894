// Bit-packed witness -> column-major trace, in place of the transpose in front of the LDE.
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

__global__ void __launch_bounds__(256) unpack_kernel(uint64_t *__restrict__ dst, const uint64_t *__restrict__ src,
                                                     uint64_t nrows, uint64_t ncols, uint64_t words_per_row,
                                                     const uint32_t *__restrict__ col_bits)
{
    extern __shared__ uint32_t bits_sm[];
    for (uint64_t c = threadIdx.x; c < ncols; c += blockDim.x) bits_sm[c] = col_bits[c];
    __syncthreads();
    const uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nrows) return;
    const uint64_t *w = src + row * words_per_row;
    uint64_t word = words_per_row ? __ldg(w) : 0, idx = 0, off = 0;
    for (uint64_t c = 0; c < ncols; c++) {
        const uint32_t nb = bits_sm[c];
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

// bits of a packed row (host check of words_per_row)
inline uint64_t packed_bits(const uint32_t *col_bits, uint64_t ncols)
{
    uint64_t s = 0;
    for (uint64_t c = 0; c < ncols; c++) s += col_bits[c];
    return s;
}

}  // namespace unpack
