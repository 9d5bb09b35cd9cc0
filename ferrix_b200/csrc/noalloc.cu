// Allocation-free CSR SpMV with a fused dot product:
//     y = A x,   dot = x . y        (FP64, device pointers, caller's stream)
//
// Who needs it: code that may not allocate device memory at the point it
// runs — for example a solver loop that is being recorded into a CUDA graph,
// a callback or library layer that only receives memory owned by a host
// application with its own pool allocator, or a real-time loop that must not
// take the driver's allocation locks. Such callers pass every input and
// output; the only other memory this entry point uses is a fixed scratch
// array compiled into the library.
//
// Scratch: one file-scope __device__ array holding the per-CTA partial sums
// of the dot product and the CTA completion counter. Every GPU that loads the
// library holds it (about 513 KiB) until the process exits. Its size fixes
// the largest matrix: one CTA per 8 rows and at most 65,536 CTAs, so at most
// 524,288 rows; larger calls are rejected with FX_INVALID_ARGUMENT.
//
// Set-up: the first call on a device, with that device current, looks up the
// device address of the scratch array (cudaGetSymbolAddress) and caches it.
// Make that first call before any stream capture begins. Later calls only
// launch work on the given stream.
//
// Sharing: all calls on a device use the same scratch array and it keeps the
// last call's contents; each call clears the counter it relies on. Calls that
// can overlap on the GPU (different streams without ordering) race on the
// scratch and give wrong results: order them on one stream or with events.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "common.hpp"
#include "device.cuh"

namespace fx {
namespace {

constexpr int kNaRowsPerCta = 8;  // one warp per row, 256 threads
constexpr int kNaMaxCtas = 65536;
constexpr int64_t kNaMaxRows = (int64_t)kNaMaxCtas * kNaRowsPerCta;
constexpr int kNaMaxDevices = 64;

struct NoAllocScratch {
    double partial[kNaMaxCtas];
    unsigned int counter;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

std::mutex g_setup_mutex;
NoAllocScratch* g_scratch_addr[kNaMaxDevices] = {};

__global__ void __launch_bounds__(256) k_spmv_dot_noalloc(int64_t n, const int64_t* __restrict__ ip,
                                                          const int64_t* __restrict__ ind,
                                                          const double* __restrict__ val,
                                                          const double* __restrict__ x, double* __restrict__ y,
                                                          double* __restrict__ dot, NoAllocScratch* sc) {
    __shared__ double sh[8];
    __shared__ int s_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t row = (int64_t)blockIdx.x * kNaRowsPerCta + warp;  // uniform per warp
    double acc = 0.0;
    if (row < n)
        for (int64_t k = ip[row] + lane; k < ip[row + 1]; k += 32) acc += val[k] * x[ind[k]];
    acc = warp_sum(acc);
    double part = 0.0;
    if (lane == 0 && row < n) {
        y[row] = acc;
        part = x[row] * acc;
    }
    if (lane == 0) sh[warp] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kNaRowsPerCta; ++w) t += sh[w];
        sc->partial[blockIdx.x] = t;
        __threadfence();
        s_last = atomicAdd(&sc->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // fixed-order total: every thread sums a strided subset, then warp and CTA order
    double t = 0.0;
    for (int c = threadIdx.x; c < (int)gridDim.x; c += blockDim.x) t += __ldcg(&sc->partial[c]);
    t = warp_sum(t);
    if (lane == 0) sh[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < kNaRowsPerCta; ++w) tot += sh[w];
        *dot = tot;
        sc->counter = 0u;
    }
}

}  // namespace
// A kernel of this file's module (preload_kernels() loads all of the module's kernels).
const void* kernels_anchor_noalloc() { return reinterpret_cast<const void*>(&k_spmv_dot_noalloc); }

}  // namespace fx

using namespace fx;

extern "C" int fx_spmv_dot_noalloc(int device, int64_t n, const int64_t* indptr, const int64_t* indices,
                                   const double* data, const double* x, double* y, double* dot, void* stream) {
    if (n <= 0 || !indptr || !indices || !data || !x || !y || !dot) return FX_INVALID_ARGUMENT;
    if (n > kNaMaxRows) return FX_INVALID_ARGUMENT;  // beyond the scratch array: at most 524,288 rows
    // y is written while other rows still read x: the two must not overlap
    const uintptr_t xb = reinterpret_cast<uintptr_t>(x), yb = reinterpret_cast<uintptr_t>(y);
    const uintptr_t nbytes = (uintptr_t)n * sizeof(double);
    if (xb < yb + nbytes && yb < xb + nbytes) return FX_INVALID_ARGUMENT;
    // an error left pending by the caller's own earlier CUDA calls is reported, not consumed
    if (cudaPeekAtLastError() != cudaSuccess) return FX_CUDA;
    if (device < 0 || device >= kNaMaxDevices) return FX_INVALID_ARGUMENT;
    int current = -1;
    if (cudaGetDevice(&current) != cudaSuccess) return FX_CUDA;
    if (current != device && cudaSetDevice(device) != cudaSuccess) return FX_CUDA;
    NoAllocScratch* sc = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_addr[device]) {
            void* addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (e != cudaSuccess || !addr) {
                if (current != device) cudaSetDevice(current);
                return FX_CUDA;
            }
            g_scratch_addr[device] = static_cast<NoAllocScratch*>(addr);
        }
        sc = g_scratch_addr[device];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = FX_OK;
    // the completion counter must start at zero even if an earlier call stopped early
    if (cudaMemsetAsync(&sc->counter, 0, sizeof(unsigned int), s) != cudaSuccess) rc = FX_CUDA;
    if (rc == FX_OK) {
        const unsigned grid = (unsigned)((n + kNaRowsPerCta - 1) / kNaRowsPerCta);
        k_spmv_dot_noalloc<<<grid, 32 * kNaRowsPerCta, 0, s>>>(n, indptr, indices, data, x, y, dot, sc);
        if (cudaGetLastError() != cudaSuccess) rc = FX_CUDA;  // no error was pending: this launch's own
    }
    if (current != device) cudaSetDevice(current);
    return rc;
}
