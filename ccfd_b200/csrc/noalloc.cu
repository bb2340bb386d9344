// Allocation-free global residual.
//
// Some callers cannot allocate device memory: a host application that hands
// its whole device heap to its own pool allocator and forbids allocations
// behind its back, or a serving loop that has already committed the device
// memory budget to resident solver states and must not fail (or stall on an
// allocation) in the middle of a request.  This entry point lets them compute
// the global residual of a residual field they already hold in device
// memory without any allocation by this library: the per-block partial sums
// live in a fixed-size file-scope __device__ array.
//
// Scratch: CCFD_NOALLOC_MAX_CELLS / 256 partial sums of 4 doubles (128 KB),
// held by every device that loads the library until the process exits.
// Every call shares it and overwrites the partials it uses before reading
// them, so nothing must be cleared between calls; calls that overlap on the
// GPU (different streams, or threads issuing concurrently) race on it.
#include <cuda_runtime.h>
#include <math.h>

#include <mutex>

#include "ccfd_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr long kMaxBlocks = CCFD_NOALLOC_MAX_CELLS / kThreads;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_partial[kMaxBlocks * 4];

// device address of g_partial, looked up once per device with that device
// current (the host-side symbol is only a stand-in, never a device address).
// It stays valid while the device's context lives, so a device must not be
// reset while the library is loaded.
double* g_partial_addr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

int scratch_for_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CCFD_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partial_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_partial) != cudaSuccess || !p) return CCFD_ERR_CUDA;
        g_partial_addr[dev] = static_cast<double*>(p);
    }
    *out = g_partial_addr[dev];
    return CCFD_OK;
}

// per-block sums of area * u_t^2, one block per 256 cells
__global__ void __launch_bounds__(kThreads) k_res_partial(const double* __restrict__ u_t,
                                                          const double* __restrict__ area, long n,
                                                          double* __restrict__ partial) {
    __shared__ double sh[4][kThreads / 32];
    long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double r[4] = {0.0, 0.0, 0.0, 0.0};
    if (c < n) {
        double a = area[c];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            double u = u_t[4 * c + v];
            r[v] = a * u * u;
        }
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r[v] += __shfl_down_sync(0xffffffffu, r[v], o);
    if (lane == 0)
#pragma unroll
        for (int v = 0; v < 4; ++v) sh[v][warp] = r[v];
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) s += sh[threadIdx.x][w];
        partial[4 * blockIdx.x + threadIdx.x] = s;
    }
}

// fixed-order sum of the partials, res = sqrt(sum * totalArea_q)
__global__ void __launch_bounds__(kThreads) k_res_final(const double* __restrict__ partial, int nb,
                                                        double total_area_q, double* __restrict__ res) {
    __shared__ double sh[4][kThreads];
    double r[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int v = 0; v < 4; ++v) r[v] += partial[4 * b + v];
#pragma unroll
    for (int v = 0; v < 4; ++v) sh[v][threadIdx.x] = r[v];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
#pragma unroll
            for (int v = 0; v < 4; ++v) sh[v][threadIdx.x] += sh[v][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 4) res[threadIdx.x] = sqrt(sh[threadIdx.x][0] * total_area_q);
}

}  // namespace

extern "C" int ccfd_global_residual_noalloc(const double* u_t, const double* area, long n_cells,
                                            double total_area_q, double* res, void* stream) {
    if (!u_t || !area || !res || n_cells <= 0) return CCFD_ERR_ARG;
    if (n_cells > CCFD_NOALLOC_MAX_CELLS) return CCFD_ERR_ARG;  // beyond the static scratch
    double* partial = nullptr;
    int st = scratch_for_current_device(&partial);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int nb = (int)((n_cells + kThreads - 1) / kThreads);
    k_res_partial<<<nb, kThreads, 0, s>>>(u_t, area, n_cells, partial);
    k_res_final<<<1, kThreads, 0, s>>>(partial, nb, total_area_q, res);
    return cudaGetLastError() == cudaSuccess ? CCFD_OK : CCFD_ERR_CUDA;
}
