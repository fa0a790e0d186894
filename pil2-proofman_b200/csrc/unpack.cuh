// Bit-packed (and indexed) witness -> column-major trace, in place of the transpose in front of
// the LDE.
//
// Format (the reference's PackedInfo, starks_gpu.cu:49-185): every row is `words_per_row` u64
// words holding its columns back to back, column c taking col_bits[c] bits, least significant
// bit first; a field may cross a word boundary.  An indexed row starts with an `index_bits`-wide
// instruction index, and the columns flagged as table columns are read instead from entry
// `index` of a shared instruction table (same packing, words_per_entry words per entry, the table
// columns in column order); an index past the table selects entry 0.
//
// Method: a column's bit position inside its stream is the sum of the widths of the earlier
// columns of the same stream, so each CTA first turns the column widths into bit positions with
// a block-wide prefix sum in shared memory (row stream and table stream at once, as the two
// 32-bit halves of one 64-bit scan).  Every field is then independent: word position >> 6, shift
// position & 63, one or two loads and a funnel shift.  One thread per row; thread i of a CTA
// writes row base+i of each column, so the column-major stores are coalesced.
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

// Column descriptions in device memory: width | source << 32 per column (the streaming slot's
// width region).
struct InfoDev {
    const uint64_t *p;
};

__device__ __forceinline__ uint64_t col_desc(const ColBytes &t, uint32_t c)
{
    const uint32_t b = t.v[c];
    return (uint64_t)(b & 127u) | ((uint64_t)(b >> 7) << 32);
}
__device__ __forceinline__ uint64_t col_desc(const InfoDev &t, uint32_t c) { return __ldg(t.p + c); }

// Bits [pos, pos + nb) of the stream `w` (1 <= nb <= 64), least significant first.  The second
// word is read only when the field crosses into it, so a field ending on the last word of the
// stream reads nothing past it.
__device__ __forceinline__ uint64_t field(const uint64_t *__restrict__ w, uint32_t pos, uint32_t nb)
{
    const uint32_t wi = pos >> 6, sh = pos & 63;
    uint64_t v = __ldg(w + wi) >> sh;
    if (sh + nb > 64) v |= __ldg(w + wi + 1) << (64 - sh);  // sh >= 1 here
    return nb < 64 ? v & ((1ull << nb) - 1) : v;
}

// Bit positions of columns [0, nc) into pos[]: bits 0-19 the position within the column's
// stream (the row stream starts after the index), bits 20-25 width - 1, bit 26 the source.
// Block-wide exclusive prefix sum of (row width, table width) pairs packed in 64 bits: every
// thread sums a contiguous run of columns, the run totals are scanned across the warp and the
// warps, and each thread writes its run's positions.  Ends with a barrier.
template <class Info>
__device__ __forceinline__ void column_positions(uint32_t *pos, const Info &info, uint32_t nc, uint32_t index_bits)
{
    __shared__ uint64_t warp_tot[32];
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5, nwarps = (blockDim.x + 31) >> 5;
    const uint32_t per = (nc + blockDim.x - 1) / blockDim.x;
    const uint32_t a = min(nc, t * per), b = min(nc, a + per);
    auto pair = [&](uint32_t c) {
        const uint64_t d = col_desc(info, c), w = d & 0xffffffffull;
        return (d >> 32) ? (w << 32) : w;
    };
    uint64_t run = 0;
    for (uint32_t c = a; c < b; c++) run += pair(c);
    uint64_t inc = run;  // inclusive scan of the run totals within the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= (uint32_t)d) inc += y;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint64_t v = lane < nwarps ? warp_tot[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= (uint32_t)d) v += y;
        }
        warp_tot[lane] = v;  // inclusive over warps
    }
    __syncthreads();
    uint64_t acc = inc - run + (warp ? warp_tot[warp - 1] : 0);  // exclusive start of this run
    for (uint32_t c = a; c < b; c++) {
        const uint64_t d = col_desc(info, c);
        const uint32_t src = (uint32_t)(d >> 32) & 1u, w = (uint32_t)d;
        const uint32_t p = src ? (uint32_t)(acc >> 32) : (uint32_t)acc + index_bits;
        pos[c] = p | ((w - 1) << 20) | (src << 26);
        acc += pair(c);
    }
    __syncthreads();
}

// Columns [c0, c0 + cc) of every row into cc column-major columns of dst (stride nrows).  A plain
// packed witness is the case index_bits = 0 with no table columns.  Dynamic shared memory:
// (c0 + cc) * 4 bytes.
template <class Info>
__global__ void __launch_bounds__(256) bitfield_unpack_kernel(uint64_t *__restrict__ dst,
                                                              const uint64_t *__restrict__ rows,
                                                              const uint64_t *__restrict__ table, uint64_t nrows,
                                                              uint64_t words_per_row, uint64_t words_per_entry,
                                                              uint64_t num_entries, uint32_t index_bits,
                                                              const __grid_constant__ Info info, uint32_t c0,
                                                              uint32_t cc)
{
    extern __shared__ uint32_t pos[];
    column_positions(pos, info, c0 + cc, index_bits);
    const uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nrows) return;
    const uint64_t *r = rows + row * words_per_row;
    const uint64_t *t = nullptr;
    if (table) {
        uint64_t index = index_bits ? field(r, 0, index_bits) : 0;
        if (index >= num_entries) index = 0;
        t = table + index * words_per_entry;
    }
    for (uint32_t c = c0; c < c0 + cc; c++) {
        const uint32_t p = pos[c];
        dst[(uint64_t)(c - c0) * nrows + row] = field((p >> 26) ? t : r, p & 0xfffffu, ((p >> 20) & 63u) + 1);
    }
}

// Launch over N rows; the dynamic shared memory holds the positions of columns [0, c0 + cc).
template <class Info>
inline cudaError_t launch(uint64_t *dst, const uint64_t *rows, const uint64_t *table, uint64_t nrows,
                          uint64_t words_per_row, uint64_t words_per_entry, uint64_t num_entries, uint32_t index_bits,
                          const Info &info, uint32_t c0, uint32_t cc, cudaStream_t s)
{
    if (cc == 0 || nrows == 0) return cudaSuccess;
    const size_t smem = (size_t)(c0 + cc) * 4;
    if (smem > 48 * 1024) return cudaErrorInvalidValue;
    bitfield_unpack_kernel<Info><<<(unsigned)((nrows + 255) / 256), 256, smem, s>>>(
        dst, rows, table, nrows, words_per_row, words_per_entry, num_entries, index_bits, info, c0, cc);
    return cudaGetLastError();
}

// bits of a packed row (host check of words_per_row)
inline uint64_t packed_bits(const uint32_t *col_bits, uint64_t ncols)
{
    uint64_t s = 0;
    for (uint64_t c = 0; c < ncols; c++) s += col_bits[c];
    return s;
}

}  // namespace unpack
