// noalloc.cu -- ippi_mass_noalloc: the deterministic FP64 mass sum of a
// density field without any device allocation.
//
// Who needs it: callers that may not allocate device memory at the point
// where they want the checksum -- hosts whose device memory is owned by
// another allocator (a framework's caching allocator, a fixed arena set up
// at start-up) and real-time loops that forbid allocation after
// initialisation.  ippi_forces() computes the same sum but needs a lattice
// handle, which allocates its own reduction scratch.
//
// The scratch is a file-scope __device__ array of kMaxRows doubles (128 KiB):
// one partial sum per lattice row.  Every GPU that loads the library holds it
// until the process exits.  The rows of one call overwrite entries 0..ny-1
// before the final pass reads them, so nothing has to start at zero; entries
// beyond ny keep whatever an earlier call left there and are never read.
// All calls share the array: calls that overlap on the GPU (on different
// streams, or from different host threads) race on it.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/ippi_lbm.h"

namespace {

constexpr int kMaxRows = IPPI_NOALLOC_MAX_ROWS;
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_row_partials[kMaxRows];

// per-device address of g_row_partials, looked up once per device and kept:
// valid while the device's primary context lives, which this library
// assumes is the whole process (no cudaDeviceReset between calls)
double* g_scratch[kMaxDevices] = {};
std::mutex g_mu;

__device__ double block_sum(double v, double* red)
{
    red[threadIdx.x] = v;
    __syncthreads();
    for (int w = kThreads / 2; w; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    return red[0];
}

// pass 1: one block per row writes that row's sum
__global__ void __launch_bounds__(kThreads) row_sums(const double* rho, int nx, double* part)
{
    __shared__ double red[kThreads];
    const double* row = rho + (long long)blockIdx.x * nx;
    double s = 0.0;
    for (int x = threadIdx.x; x < nx; x += kThreads) s += row[x];
    const double r = block_sum(s, red);
    if (threadIdx.x == 0) part[blockIdx.x] = r;
}

// pass 2: one block adds the row sums in a fixed order
__global__ void __launch_bounds__(kThreads) final_sum(const double* part, int ny, double* out)
{
    __shared__ double red[kThreads];
    double s = 0.0;
    for (int y = threadIdx.x; y < ny; y += kThreads) s += part[y];
    const double r = block_sum(s, red);
    if (threadIdx.x == 0) *out = r;
}

}  // namespace

extern "C" int ippi_mass_noalloc(const double* rho, int nx, int ny, double* mass, void* stream)
{
    if (!rho || !mass) return IPPI_ERR_ARG;
    if (nx < 1 || ny < 1) return IPPI_ERR_ARG;
    if (ny > kMaxRows) {
        fprintf(stderr, "ippi_mass_noalloc: ny = %d exceeds the %d rows of its fixed scratch\n", ny,
                kMaxRows);
        return IPPI_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return IPPI_ERR_CUDA;
    double* part;
    {
        // set-up, once per device, with that device current: the device
        // address of the scratch array (host code cannot use the symbol itself)
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_row_partials) != cudaSuccess || !p) return IPPI_ERR_CUDA;
            g_scratch[dev] = static_cast<double*>(p);
        }
        part = g_scratch[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // an error pending from the caller's earlier launches is theirs: leave
    // it pending, and do not launch behind it
    if (cudaPeekAtLastError() != cudaSuccess) return IPPI_ERR_CUDA;
    row_sums<<<ny, kThreads, 0, st>>>(rho, nx, part);
    if (cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();  // this call's launch failed: clear its error
        return IPPI_ERR_CUDA;
    }
    final_sum<<<1, kThreads, 0, st>>>(part, ny, mass);
    if (cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();
        return IPPI_ERR_CUDA;
    }
    return IPPI_OK;
}
