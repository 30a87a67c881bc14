/*
 * php_noalloc.cu -- field maxima without any device allocation.
 *
 * php_diagnostics reduces |E| and |Ex| in two passes through a scratch
 * buffer that php_create allocates.  Some callers cannot allocate device
 * memory when they need these maxima:
 *   - a divergence or health check that runs when HBM is exhausted (many
 *     resident domains, or one large domain with its lattice state, fill
 *     most of the 180 GB), where one more cudaMalloc is exactly what fails;
 *     a domain above PHP_NOALLOC_MAX_CELLS (2^26 cells) is reduced in
 *     pieces of at most that many cells, one call per piece, the caller
 *     keeping the larger results;
 *   - hosts whose allocator owns all device memory (a framework caching
 *     allocator, a fixed memory pool) and forbid allocations behind its back;
 *   - latency-critical loops, where cudaMalloc/cudaFree would synchronise the
 *     device.
 * php_field_maxima_noalloc serves them: the block partials live in the
 * file-scope array below, which every GPU that loads this library holds
 * (256 KB) until the process exits.
 */
#include "php_fdtd.h"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>

namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 16;
constexpr int64_t kCellsPerBlock = (int64_t)kThreads * kCellsPerThread;
constexpr int kMaxBlocks = PHP_NOALLOC_MAX_CELLS / (int)(kThreads * kCellsPerThread);
constexpr int kMaxDevices = 64;
/* pass 1 writes one partial per kCellsPerBlock cells: the cap must be a
 * whole number of blocks, or its last block would write past the array */
static_assert(PHP_NOALLOC_MAX_CELLS % kCellsPerBlock == 0, "PHP_NOALLOC_MAX_CELLS must be a multiple of 4096");

/* One partial (max |E|, max |Ex|) per block of the first pass.  Pass 1
 * writes every entry that pass 2 reads, so nothing needs clearing between
 * calls; calls that overlap on the GPU (two streams at once) race on it. */
static __device__ __align__(256) double g_partials[kMaxBlocks][2];

/* The device address of g_partials, per device, with the id of the CUDA
 * context it was resolved in: a context destroyed and made anew (a
 * cudaDeviceReset by the caller) gets a new id, and the address is looked up
 * again in it. */
struct Resolved {
    unsigned long long ctx_id = 0;
    double (*ptr)[2] = nullptr;
};
std::mutex g_mu;
Resolved g_resolved[kMaxDevices];

typedef CUresult (*ctx_current_fn)(CUcontext*);
typedef CUresult (*ctx_id_fn)(CUcontext, unsigned long long*);

/* id of the context current on this thread; false if there is none yet */
static bool current_ctx_id(unsigned long long* id)
{
    static ctx_current_fn get_current = nullptr;
    static ctx_id_fn get_id = nullptr;
    if (!get_current || !get_id) {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            qa != cudaDriverEntryPointSuccess || !a ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qb != cudaDriverEntryPointSuccess || !b)
            return false;
        get_current = reinterpret_cast<ctx_current_fn>(a);
        get_id = reinterpret_cast<ctx_id_fn>(b);
    }
    CUcontext c = nullptr;
    if (get_current(&c) != CUDA_SUCCESS || !c) return false;
    return get_id(c, id) == CUDA_SUCCESS;
}

/* sqrt(Ex^2 + Ey^2 + Ez^2) in the order of fdtd.c:3542-3544 and |Ex|; the
 * comparisons skip NaN as the reference's `>` tests do. */
__global__ void __launch_bounds__(kThreads) noalloc_pass1(const double* __restrict__ ex, const double* __restrict__ ey,
                                                          const double* __restrict__ ez, int64_t n,
                                                          double (*partials)[2])
{
    double me = 0.0, mx = 0.0;
    const int64_t base = (int64_t)blockIdx.x * kCellsPerBlock + threadIdx.x;
#pragma unroll 4
    for (int q = 0; q < kCellsPerThread; ++q) {
        const int64_t t = base + (int64_t)q * kThreads;
        if (t < n) {
            const double x = ex[t], y = ey[t], z = ez[t];
            const double e = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
            if (e > me) me = e;
            const double ax = fabs(x);
            if (ax > mx) mx = ax;
        }
    }
    __shared__ double se[kThreads], sx[kThreads];
    se[threadIdx.x] = me;
    sx[threadIdx.x] = mx;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            se[threadIdx.x] = fmax(se[threadIdx.x], se[threadIdx.x + w]);
            sx[threadIdx.x] = fmax(sx[threadIdx.x], sx[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[blockIdx.x][0] = se[0];
        partials[blockIdx.x][1] = sx[0];
    }
}

__global__ void __launch_bounds__(kThreads) noalloc_pass2(const double (*partials)[2], int nblocks, double* out2)
{
    double me = 0.0, mx = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += kThreads) {
        me = fmax(me, partials[b][0]);
        mx = fmax(mx, partials[b][1]);
    }
    __shared__ double se[kThreads], sx[kThreads];
    se[threadIdx.x] = me;
    sx[threadIdx.x] = mx;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            se[threadIdx.x] = fmax(se[threadIdx.x], se[threadIdx.x + w]);
            sx[threadIdx.x] = fmax(sx[threadIdx.x], sx[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out2[0] = se[0];
        out2[1] = sx[0];
    }
}

} // namespace

extern "C" int php_field_maxima_noalloc(const double* ex, const double* ey, const double* ez, int64_t n, double* out2,
                                        void* stream)
{
    if (!out2 || n < 0 || (n > 0 && (!ex || !ey || !ez))) return PHP_ERR_INPUT;
    if (n > PHP_NOALLOC_MAX_CELLS) return PHP_ERR_INPUT;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PHP_ERR_CUDA;
    double(*partials)[2] = nullptr;
    {
        /* first call on this device, or in a new context of it: resolve the
         * device address of the file-scope array (its host-side name is only
         * a stand-in), with the device current */
        std::lock_guard<std::mutex> lock(g_mu);
        unsigned long long id = 0;
        const bool known = current_ctx_id(&id);
        Resolved& r = g_resolved[dev];
        if (!known || !r.ptr || r.ctx_id != id) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_partials) != cudaSuccess || !p) return PHP_ERR_CUDA;
            if (!current_ctx_id(&id)) return PHP_ERR_CUDA;
            r.ptr = reinterpret_cast<double(*)[2]>(p);
            r.ctx_id = id;
        }
        partials = r.ptr;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nblocks = (int)((n + kCellsPerBlock - 1) / kCellsPerBlock);
    if (nblocks > 0) noalloc_pass1<<<nblocks, kThreads, 0, s>>>(ex, ey, ez, n, partials);
    noalloc_pass2<<<1, kThreads, 0, s>>>(partials, nblocks, out2);
    return cudaGetLastError() == cudaSuccess ? PHP_OK : PHP_ERR_CUDA;
}
