// Row-major trace -> column-major columns with the row tiles staged by the Tensor Memory
// Accelerator (the reference's fromRowMajorToColMajor, goldilocks_tooling.cu:28-59, which moves
// one element per thread).
//
// One CTA of 32 x 8 threads moves a 32-row x 32-column tile.  Thread 0 arms an mbarrier with the
// tile's byte count and issues two 2-D bulk tensor loads (cp.async.bulk.tensor, boxes of 32 rows x
// 16 columns = 128-byte rows) into shared memory; the copies bypass the registers and complete on
// the barrier.  The boxes use the 128-byte swizzle: the 16-byte chunk j of box row r lands at chunk
// j ^ (r & 7), so the transposed read (lanes along the rows of one column) touches eight different
// chunk positions instead of one bank.  Every thread then writes 4 columns x 32 consecutive rows:
// 256-byte coalesced stores.  Out-of-range rows and columns of edge tiles are zero-filled by the
// copy and skipped by the stores.  The wait on the barrier is bounded: if the copy never lands the
// CTA records an error flag and returns instead of spinning.
//
// Preconditions (checked by the host dispatcher, which otherwise uses ntt::transpose_kernel): the
// source 16-byte aligned, its row pitch nCols * 8 a multiple of 16 bytes (nCols even), and the
// driver's cuTensorMapEncodeTiled available.  Tile coordinates are multiples of 32 elements, so
// every copy starts on a 16-byte boundary.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "prof.cuh"

__device__ int g_tma_error;  // set when a tile copy did not land within the wait bound

namespace ntt {

constexpr uint32_t TMA_WAIT_LIMIT = 1u << 22;  // try_wait rounds before a CTA gives up

__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity)
{
    for (uint32_t i = 0; i < TMA_WAIT_LIMIT; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(256) transpose_tma_kernel(uint64_t *__restrict__ dst,
                                                            const __grid_constant__ CUtensorMap src_map,
                                                            uint64_t nrows, uint64_t ncols, uint64_t dst_cs)
{
    __shared__ __align__(1024) uint64_t box[2][32][16];  // two boxes: columns 0-15 and 16-31 of the tile
    __shared__ __align__(8) uint64_t mbar_storage;
    const uint32_t tx = threadIdx.x, ty = threadIdx.y;
    const uint64_t r0 = (uint64_t)blockIdx.x * 32, c0 = (uint64_t)blockIdx.y * 32;
    const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&mbar_storage);
    if (tx == 0 && ty == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(2u * 32u * 16u * 8u)
                     : "memory");
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const uint32_t dst_smem = (uint32_t)__cvta_generic_to_shared(&box[b][0][0]);
            const int x = (int)(c0 + 16 * b), y = (int)r0;  // x: column (multiple of 16 elements), y: row
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                "[%4];" ::"r"(dst_smem),
                "l"(reinterpret_cast<uint64_t>(&src_map)), "r"(x), "r"(y), "r"(mbar)
                : "memory");
        }
    }
    __syncthreads();  // the barrier is initialised before anyone waits on it
    if (!mbar_wait_bounded(mbar, 0)) {
        if (tx == 0 && ty == 0) atomicExch(&g_tma_error, 1);
        return;
    }
    const uint64_t r = r0 + tx;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint32_t c = ty + 8 * j;  // tile column 0..31
        const uint32_t b = c >> 4, cc = c & 15;
        const uint32_t chunk = (cc >> 1) ^ (tx & 7);
        const uint64_t v = *reinterpret_cast<const uint64_t *>(reinterpret_cast<const unsigned char *>(&box[b][tx][0]) +
                                                             (chunk << 4) + ((cc & 1) << 3));
        if (r < nrows && c0 + c < ncols) dst[(c0 + c) * dst_cs + r] = v;
    }
}

// cuTensorMapEncodeTiled from the driver, looked up once (null when the driver does not offer it)
inline PFN_cuTensorMapEncodeTiled tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled)p;
        cudaGetLastError();
    });
    return fn;
}

// The 2-D tensor map of a row-major nrows x ncols source: boxes of 32 rows x 16 columns, 128-byte
// swizzle, zero fill outside the matrix.  False when the shape or alignment does not allow TMA.
inline bool tma_source_map(CUtensorMap *map, const uint64_t *src, uint64_t nrows, uint64_t ncols)
{
    if (((uintptr_t)src & 15) || (ncols & 1) || ncols == 0 || nrows == 0 || nrows > (1ull << 31) ||
        ncols > (1ull << 31))
        return false;
    PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {ncols, nrows};
    const cuuint64_t strides[1] = {ncols * 8};
    const cuuint32_t boxdim[2] = {16, 32};
    const cuuint32_t estrides[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<uint64_t *>(src), dims, strides, boxdim, estrides,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace ntt
