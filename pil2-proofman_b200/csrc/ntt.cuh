// Low-degree extension of Goldilocks columns on the device.
//
// out[j] = p(7 * w_NExt^j), where p interpolates the column on <w_N> and w_k is the
// reference's W[log2 k] (goldilocks_base_field.cpp:11-44); NTT_Goldilocks::LDE
// (ntt_goldilocks.cpp:369-404) is the CPU statement of the same map.
//
// Data layout: columns are contiguous (column-major, element (row, col) at col*stride + row).
// Plan for one column of N = 2^lg rows and blowup B = 2^b:
//   1. inverse DIF NTT of size N (natural in, bit-reversed out), in windows of <= 12 bits;
//      the last window scales position p by N^-1 * 7^bitrev(p), so position p then holds
//      coefficient c_i * 7^i with i = bitrev(p);
//   2. forward DIT NTT of size N*B (bit-reversed in, natural out).  In bit-reversed order
//      the zero-padded coefficient vector is nonzero only at multiples of B, and its first
//      b butterfly stages just copy, so the first window reads position P from p = P >> b
//      and starts at stage b.  The last window writes canonical values.
// A window covering butterfly stages [s0, s0+k) is a batch of independent 2^k-point
// transforms over elements at stride 2^s0.  One CTA loads a 2^k x L tile (L consecutive
// low-index lanes) into shared memory, runs the k radix-2 stages there with twiddles
// w_{2^(t+1)}^j from a 2048-entry table, and applies the single inter-window twiddle
// w_{2^(s0+k)}^(bitrev_k(mid)*lo) per element (before a DIT window, after a DIF window),
// formed from a two-level table of w_{2^26} powers.
#pragma once
#include "gl64.cuh"
#include "prof.cuh"

#define NTT_KMAX 12   // widest window: inner twiddles w_{2^12}^j, j < 2048
#define NTT_TWLG 26   // inter-window twiddles: powers of w_{2^26}; transforms up to 2^26 points
#define NTT_TILE_MAX 8192

__device__ uint64_t g_ntt_inner_fwd[1 << (NTT_KMAX - 1)];
__device__ uint64_t g_ntt_inner_inv[1 << (NTT_KMAX - 1)];
__device__ uint64_t g_ntt_tw_lo_fwd[1 << 13];
__device__ uint64_t g_ntt_tw_hi_fwd[1 << 13];
__device__ uint64_t g_ntt_tw_lo_inv[1 << 13];
__device__ uint64_t g_ntt_tw_hi_inv[1 << 13];
__device__ uint64_t g_ntt_sh_lo[1 << 12];  // 7^j
__device__ uint64_t g_ntt_sh_hi[1 << 14];  // 7^(4096 j)

namespace ntt {

enum { POST_NONE = 0, POST_COSET = 1, POST_CANON = 2 };

struct Pass {
    const uint64_t *src;
    uint64_t *dst;
    uint64_t src_cs, dst_cs;  // column strides, elements
    uint64_t ninv;            // N^-1 for POST_COSET
    uint32_t lg;              // log2 of the transform length (dst positions)
    uint32_t s0, k, lgL;      // window: stages [s0, s0+k), 2^lgL lanes per tile
    uint32_t rep;             // source position = dst position >> rep
    uint32_t dif;             // 1: inverse DIF window, 0: forward DIT window
    uint32_t post;            // POST_*
};

__device__ __forceinline__ uint32_t brev_bits(uint32_t x, uint32_t bits)
{
    return bits ? (__brev(x) >> (32 - bits)) : 0u;
}

__device__ __forceinline__ uint64_t big_twiddle(uint64_t e, bool inv)
{
    const uint64_t *lo = inv ? g_ntt_tw_lo_inv : g_ntt_tw_lo_fwd;
    const uint64_t *hi = inv ? g_ntt_tw_hi_inv : g_ntt_tw_hi_fwd;
    return gl::mul(__ldg(lo + (e & 8191)), __ldg(hi + (e >> 13)));
}

__global__ void __launch_bounds__(512) pass_kernel(Pass a)
{
    extern __shared__ uint64_t sm[];
    const uint32_t k = a.k, lgL = a.lgL, s0 = a.s0;
    const uint32_t T = 1u << (k + lgL);
    const uint32_t Lm = (1u << lgL) - 1;
    const uint32_t nlob = s0 - lgL;
    const uint64_t tile = blockIdx.x;
    const uint64_t hi = tile >> nlob;
    const uint64_t lob = tile & ((1ull << nlob) - 1);
    const uint64_t base = (hi << (s0 + k)) | (lob << lgL);
    const uint64_t *S = a.src + (uint64_t)blockIdx.y * a.src_cs;
    uint64_t *D = a.dst + (uint64_t)blockIdx.y * a.dst_cs;
    const bool inv = a.dif != 0;
    const uint32_t tw_shift = NTT_TWLG - s0 - k;

    for (uint32_t q = threadIdx.x; q < T; q += blockDim.x) {
        const uint64_t pos = base | ((uint64_t)(q >> lgL) << s0) | (q & Lm);
        uint64_t v = S[pos >> a.rep];
        if (!inv && s0 > 0) {
            const uint64_t lo = (lob << lgL) | (q & Lm);
            const uint64_t E = (uint64_t)brev_bits(q >> lgL, k) * lo;
            if (E) v = gl::mul(v, big_twiddle(E << tw_shift, false));
        }
        sm[q] = v;
    }
    __syncthreads();

    const uint64_t *inner = inv ? g_ntt_inner_inv : g_ntt_inner_fwd;
    const uint32_t nbf = T >> 1;
    for (uint32_t step = 0; step < k; step++) {
        const uint32_t t = inv ? (k - 1 - step) : step;
        const uint32_t h = 1u << t;
        for (uint32_t b = threadIdx.x; b < nbf; b += blockDim.x) {
            const uint32_t l = b & Lm, mm = b >> lgL;
            const uint32_t m = ((mm >> t) << (t + 1)) | (mm & (h - 1));
            const uint32_t i1 = (m << lgL) | l, i2 = i1 + (h << lgL);
            uint64_t u = sm[i1], v = sm[i2];
            if (!inv) {
                if (t) v = gl::mul(v, __ldg(inner + ((m & (h - 1)) << (NTT_KMAX - 1 - t))));
                sm[i1] = gl::add(u, v);
                sm[i2] = gl::sub(u, v);
            } else {
                sm[i1] = gl::add(u, v);
                uint64_t d = gl::sub(u, v);
                if (t) d = gl::mul(d, __ldg(inner + ((m & (h - 1)) << (NTT_KMAX - 1 - t))));
                sm[i2] = d;
            }
        }
        __syncthreads();
    }

    for (uint32_t q = threadIdx.x; q < T; q += blockDim.x) {
        const uint64_t pos = base | ((uint64_t)(q >> lgL) << s0) | (q & Lm);
        uint64_t v = sm[q];
        if (inv && s0 > 0) {
            const uint64_t lo = (lob << lgL) | (q & Lm);
            const uint64_t E = (uint64_t)brev_bits(q >> lgL, k) * lo;
            if (E) v = gl::mul(v, big_twiddle(E << tw_shift, true));
        }
        if (a.post == POST_COSET) {
            const uint32_t br = brev_bits((uint32_t)pos, a.lg);
            const uint64_t f = gl::mul(__ldg(g_ntt_sh_lo + (br & 4095)), __ldg(g_ntt_sh_hi + (br >> 12)));
            v = gl::mul(v, gl::mul(f, a.ninv));
        } else if (a.post == POST_CANON) {
            v = gl::canon(v);
        }
        D[pos] = v;
    }
}

// row-major (nrows x ncols) -> column-major with column stride dst_cs
__global__ void __launch_bounds__(256) transpose_kernel(uint64_t *__restrict__ dst, const uint64_t *__restrict__ src,
                                                        uint64_t nrows, uint64_t ncols, uint64_t dst_cs)
{
    __shared__ uint64_t tile[32][33];
    const uint64_t r0 = (uint64_t)blockIdx.x * 32, c0 = (uint64_t)blockIdx.y * 32;
    const uint32_t tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint64_t r = r0 + ty + 8 * j, c = c0 + tx;
        if (r < nrows && c < ncols) tile[ty + 8 * j][tx] = src[r * ncols + c];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint64_t c = c0 + ty + 8 * j, r = r0 + tx;
        if (r < nrows && c < ncols) dst[c * dst_cs + r] = tile[tx][ty + 8 * j];
    }
}

// ------------------------------------------------------------------ host side ----

struct Window {
    uint32_t s0, k, lgL;
};

// Windows covering stages [lo, hi).  The window that starts at `lo` keeps every lower lane
// (lgL = lo) so its tile is one contiguous run; the others take 8 lanes (4 for 11-bit windows).
inline int plan_windows(uint32_t lo, uint32_t hi, Window *w, int maxw)
{
    int n = 0;
    uint32_t total = hi - lo;
    uint32_t k0 = total;
    if (k0 > NTT_KMAX) k0 = NTT_KMAX;
    if (k0 + lo > 13) k0 = (lo >= 13) ? 0 : 13 - lo;
    if (k0 == 0 && total > 0) return -1;  // stage offset too large for one tile
    w[n++] = Window{lo, k0, lo};
    uint32_t rest = total - k0, s = lo + k0;
    uint32_t np = (rest + 10) / 11;
    for (uint32_t i = 0; i < np; i++) {
        uint32_t k = rest / (np - i) + ((rest % (np - i)) ? 1 : 0);
        uint32_t lgL = k >= 11 ? 2 : 3;
        if (lgL > s) lgL = s;
        if (n >= maxw) return -1;
        w[n++] = Window{s, k, lgL};
        s += k;
        rest -= k;
    }
    return n;
}

inline cudaError_t launch_pass(const Pass &p, uint64_t ncols, cudaStream_t stream)
{
    const uint32_t T = 1u << (p.k + p.lgL);
    const uint64_t tiles = (1ull << p.lg) >> (p.k + p.lgL);
    uint32_t threads = T / 2;
    if (threads < 32) threads = 32;
    if (threads > 512) threads = 512;
    dim3 grid((unsigned)tiles, (unsigned)ncols);
    pass_kernel<<<grid, threads, (size_t)T * 8, stream>>>(p);
    prof::count();
    return cudaGetLastError();
}

// Scratch needed by lde(): one column-major copy of the trace.
inline uint64_t lde_scratch_words(uint32_t nBits, uint64_t ncols) { return (1ull << nBits) * ncols; }

// d_lde: column-major NExt x ncols (stride NExt).  d_trace: row-major (trace_rowmajor) or
// column-major with stride N.  d_scratch: lde_scratch_words() words, distinct from both.
inline cudaError_t lde(uint64_t *d_lde, const uint64_t *d_trace, bool trace_rowmajor, uint32_t nBits,
                       uint32_t nBitsExt, uint64_t ncols, uint64_t *d_scratch, cudaStream_t stream)
{
    if (ncols == 0) return cudaSuccess;
    if (nBitsExt < nBits || nBitsExt > NTT_TWLG || ncols > 65535) return cudaErrorInvalidValue;
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    const uint32_t b = nBitsExt - nBits;
    cudaError_t err;

    const uint64_t *cur = d_trace;
    uint64_t cur_cs = N;
    if (trace_rowmajor) {
        prof::Scope ps(prof::TRANSPOSE, stream);
        dim3 grid((unsigned)((N + 31) / 32), (unsigned)((ncols + 31) / 32));
        transpose_kernel<<<grid, dim3(32, 8), 0, stream>>>(d_scratch, d_trace, N, ncols, N);
        prof::count();
        if ((err = cudaGetLastError()) != cudaSuccess) return err;
        cur = d_scratch;
    }

    // inverse DIF over [0, nBits), windows applied from the top stage down
    Window w[8];
    int nw = nBits ? plan_windows(0, nBits, w, 8) : 0;
    if (nw < 0) return cudaErrorInvalidValue;
    const uint64_t ninv = glh::inv(N % GL_P);
    {
    prof::Scope ps(prof::NTT_INV, stream);
    for (int i = nw - 1; i >= 0; i--) {
        Pass p{};
        p.src = cur;
        p.dst = d_scratch;
        p.src_cs = cur_cs;
        p.dst_cs = N;
        p.ninv = ninv;
        p.lg = nBits;
        p.s0 = w[i].s0;
        p.k = w[i].k;
        p.lgL = w[i].lgL;
        p.rep = 0;
        p.dif = 1;
        p.post = (i == 0) ? POST_COSET : POST_NONE;
        if ((err = launch_pass(p, ncols, stream)) != cudaSuccess) return err;
        cur = d_scratch;
        cur_cs = N;
    }
    }

    // forward DIT over [b, nBitsExt) with replication by 2^b on the first window
    nw = plan_windows(b, nBitsExt, w, 8);
    if (nw < 0) return cudaErrorInvalidValue;
    prof::Scope ps(prof::NTT_FWD, stream);
    for (int i = 0; i < nw; i++) {
        Pass p{};
        p.src = (i == 0) ? cur : d_lde;
        p.dst = d_lde;
        p.src_cs = (i == 0) ? cur_cs : NExt;
        p.dst_cs = NExt;
        p.ninv = 1;
        p.lg = nBitsExt;
        p.s0 = w[i].s0;
        p.k = w[i].k;
        p.lgL = w[i].lgL;
        p.rep = (i == 0) ? b : 0;
        p.dif = 0;
        p.post = (i == nw - 1) ? POST_CANON : POST_NONE;
        if ((err = launch_pass(p, ncols, stream)) != cudaSuccess) return err;
    }
    return cudaSuccess;
}

// Twiddle and coset tables, computed on the host once per device.
inline cudaError_t init_tables()
{
    static uint64_t inner_f[1 << (NTT_KMAX - 1)], inner_i[1 << (NTT_KMAX - 1)];
    static uint64_t lo_f[1 << 13], hi_f[1 << 13], lo_i[1 << 13], hi_i[1 << 13];
    static uint64_t sh_lo[1 << 12], sh_hi[1 << 14];
    static bool ready = false;
    if (!ready) {
        const uint64_t w12 = glh::root_of_unity(NTT_KMAX), w12i = glh::inv(w12);
        inner_f[0] = inner_i[0] = 1;
        for (int j = 1; j < (1 << (NTT_KMAX - 1)); j++) {
            inner_f[j] = glh::mul(inner_f[j - 1], w12);
            inner_i[j] = glh::mul(inner_i[j - 1], w12i);
        }
        const uint64_t W = glh::root_of_unity(NTT_TWLG), Wi = glh::inv(W);
        const uint64_t W13 = glh::pow(W, 1 << 13), W13i = glh::pow(Wi, 1 << 13);
        lo_f[0] = lo_i[0] = hi_f[0] = hi_i[0] = 1;
        for (int j = 1; j < (1 << 13); j++) {
            lo_f[j] = glh::mul(lo_f[j - 1], W);
            lo_i[j] = glh::mul(lo_i[j - 1], Wi);
            hi_f[j] = glh::mul(hi_f[j - 1], W13);
            hi_i[j] = glh::mul(hi_i[j - 1], W13i);
        }
        const uint64_t s4096 = glh::pow(7, 4096);
        sh_lo[0] = sh_hi[0] = 1;
        for (int j = 1; j < (1 << 12); j++) sh_lo[j] = glh::mul(sh_lo[j - 1], 7);
        for (int j = 1; j < (1 << 14); j++) sh_hi[j] = glh::mul(sh_hi[j - 1], s4096);
        ready = true;
    }
    cudaError_t e;
    if ((e = cudaMemcpyToSymbol(g_ntt_inner_fwd, inner_f, sizeof(inner_f))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_inner_inv, inner_i, sizeof(inner_i))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_tw_lo_fwd, lo_f, sizeof(lo_f))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_tw_hi_fwd, hi_f, sizeof(hi_f))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_tw_lo_inv, lo_i, sizeof(lo_i))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_tw_hi_inv, hi_i, sizeof(hi_i))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_sh_lo, sh_lo, sizeof(sh_lo))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(g_ntt_sh_hi, sh_hi, sizeof(sh_hi))) != cudaSuccess) return e;
    return cudaSuccess;
}

}  // namespace ntt
