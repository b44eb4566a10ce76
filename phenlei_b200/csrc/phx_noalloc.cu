// Allocation-free variant of the FP64 residual-monitor reduction
// (phx_residual_norm_noalloc, include/phx.h).
//
// The reduction of update_kernel / phx_residual_norm keeps its partial sums in
// a context's cudaMalloc'd Reduce record.  This variant needs no context and
// allocates nothing: its scratch is the file-scope device array below, whose
// address is looked up once per device with cudaGetSymbolAddress (the first
// call on a device does that set-up; make it before any stream capture).  Each
// call waits for its stream before it returns: the result is copied to host
// memory.
//
// Scratch contract:
//  * capacity: kNoAllocMaxBlocks x kNoAllocMaxVars partial sums (64 KiB); the
//    first pass writes every slot the second pass reads, so nothing has to
//    start at zero;
//  * one scratch per device: calls that overlap on one device (other streams
//    or host threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <math.h>
#include <mutex>

#include "phx_internal.h"

namespace phx {

static constexpr int kNoAllocMaxBlocks = 1024;
static constexpr int kNoAllocMaxVars = 8;
static constexpr int kNoAllocThreads = 256;
static constexpr int kNoAllocMaxDevices = 64;

// partial sums [block][var], then the final sums [var] after them
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxBlocks * kNoAllocMaxVars + kNoAllocMaxVars];

// Pass 1: grid-stride sum of squares of res[m * nTotal + c], c < nCell, one
// partial per block and variable.
__global__ void __launch_bounds__(kNoAllocThreads) noalloc_partial_kernel(const double *res, long long nCell,
                                                                          long long nTotal, int nvar, double *scratch)
{
    __shared__ double part[kNoAllocThreads / 32][kNoAllocMaxVars];
    double s[kNoAllocMaxVars];
#pragma unroll
    for (int m = 0; m < kNoAllocMaxVars; ++m) s[m] = 0.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nCell;
         c += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int m = 0; m < kNoAllocMaxVars; ++m) {
            if (m < nvar) {
                const double v = res[m * nTotal + c];
                s[m] += v * v;
            }
        }
    }
    const int wid = threadIdx.x >> 5, ln = threadIdx.x & 31;
#pragma unroll
    for (int m = 0; m < kNoAllocMaxVars; ++m) {
        double v = s[m];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (ln == 0) part[wid][m] = v;
    }
    __syncthreads();
    if (threadIdx.x < nvar) {
        double v = 0.0;
        for (int i = 0; i < kNoAllocThreads / 32; ++i) v += part[i][threadIdx.x];
        scratch[blockIdx.x * kNoAllocMaxVars + threadIdx.x] = v;
    }
}

// Pass 2 (one block): sums the partials, out[m] = sqrt(sum / nCell).
__global__ void __launch_bounds__(kNoAllocThreads) noalloc_final_kernel(int nblocks, int nvar, double ncell,
                                                                        double *scratch)
{
    __shared__ double part[kNoAllocThreads / 32];
    for (int m = 0; m < nvar; ++m) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += scratch[b * kNoAllocMaxVars + m];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int i = 0; i < kNoAllocThreads / 32; ++i) t += part[i];
            scratch[kNoAllocMaxBlocks * kNoAllocMaxVars + m] = sqrt(t / ncell);
        }
        __syncthreads();
    }
}

// Device address of the scratch, looked up on the first call on a device (with
// that device current) and kept; a failed lookup is not kept, so a later call
// tries again.
static double *g_noalloc_ptr[kNoAllocMaxDevices];
static std::mutex g_noalloc_mutex;

static cudaError_t noalloc_scratch(int dev, double **ptr)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return e != cudaSuccess ? e : cudaErrorInvalidSymbol;
        g_noalloc_ptr[dev] = static_cast<double *>(p);
    }
    *ptr = g_noalloc_ptr[dev];
    return cudaSuccess;
}

}  // namespace phx

extern "C" int phx_residual_norm_noalloc(const double *res_dev, int64_t n_cell, int64_t n_total, int nvar,
                                         double *out_host, void *stream)
{
    using namespace phx;
    if (!res_dev || !out_host || n_cell <= 0 || n_total < n_cell || nvar < 1) return PHX_ERR_ARG;
    if (nvar > kNoAllocMaxVars) return PHX_ERR_ARG;   // beyond the scratch's variable capacity
    // an error the calling thread left unchecked is not taken for this call's
    // own: it is reported (PHX_ERR_CUDA) and left in place, and nothing runs
    if (cudaPeekAtLastError() != cudaSuccess) return PHX_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return PHX_ERR_CUDA;
    double *scratch = nullptr;
    if (noalloc_scratch(dev, &scratch) != cudaSuccess || !scratch) return PHX_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    long long want = (n_cell + kNoAllocThreads - 1) / kNoAllocThreads;
    const int blocks = (int)(want < kNoAllocMaxBlocks ? want : kNoAllocMaxBlocks);
    noalloc_partial_kernel<<<blocks, kNoAllocThreads, 0, s>>>(res_dev, (long long)n_cell, (long long)n_total, nvar,
                                                              scratch);
    noalloc_final_kernel<<<1, kNoAllocThreads, 0, s>>>(blocks, nvar, (double)n_cell, scratch);
    if (cudaGetLastError() != cudaSuccess) return PHX_ERR_CUDA;
    if (cudaMemcpyAsync(out_host, scratch + kNoAllocMaxBlocks * kNoAllocMaxVars, sizeof(double) * nvar,
                        cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return PHX_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PHX_ERR_CUDA;
    return PHX_OK;
}
