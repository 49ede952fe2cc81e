// Platform layer: the only place that names CUDA launch / memory primitives.
// Every kernel and allocation in the library goes through these helpers.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

#define DNDSB_HD __host__ __device__ __forceinline__
#define DNDSB_D __device__ __forceinline__
#define DNDSB_GLOBAL __global__

namespace dndsb
{
using real = double;
using index_t = int64_t;

// grid-stride loop over [0, n)
#define DNDSB_KERNEL_LOOP(i, n)                                                      \
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (int64_t)(n); \
         i += (int64_t)gridDim.x * blockDim.x)

inline unsigned grid_for(int64_t n, int block)
{
    int64_t g = (n + block - 1) / block;
    if (g < 1)
        g = 1;
    if (g > 148 * 64)
        g = 148 * 64; // grid-stride loops cover the rest
    return (unsigned)g;
}

#define DNDSB_LAUNCH(kernel, n, block, stream, ...)                                              \
    do                                                                                           \
    {                                                                                            \
        if ((n) > 0)                                                                             \
            kernel<<<::dndsb::grid_for((n), (block)), (block), 0, (cudaStream_t)(stream)>>>(__VA_ARGS__); \
    } while (0)

inline cudaError_t dev_alloc(void **p, size_t bytes) { return cudaMalloc(p, bytes > 0 ? bytes : 16); }
inline void dev_free(void *p)
{
    if (p)
        cudaFree(p);
}
inline cudaError_t h2d(void *dst, const void *src, size_t bytes, cudaStream_t s) { return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s); }
inline cudaError_t d2h(void *dst, const void *src, size_t bytes, cudaStream_t s) { return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s); }
inline cudaError_t d2d(void *dst, const void *src, size_t bytes, cudaStream_t s) { return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s); }
inline cudaError_t dev_zero(void *p, size_t bytes, cudaStream_t s) { return cudaMemsetAsync(p, 0, bytes, s); }
inline cudaError_t dev_sync(cudaStream_t s) { return cudaStreamSynchronize(s); }
inline cudaError_t last_error() { return cudaGetLastError(); }
// private streams, events and captured graphs (the native linear solve)
inline cudaError_t stream_create(cudaStream_t *s) { return cudaStreamCreateWithFlags(s, cudaStreamNonBlocking); }
inline void stream_free(cudaStream_t s)
{
    if (s)
        cudaStreamDestroy(s);
}
inline cudaError_t event_create(cudaEvent_t *e) { return cudaEventCreateWithFlags(e, cudaEventDisableTiming); }
inline void event_free(cudaEvent_t e)
{
    if (e)
        cudaEventDestroy(e);
}
inline cudaError_t event_record(cudaEvent_t e, cudaStream_t s) { return cudaEventRecord(e, s); }
inline cudaError_t stream_wait(cudaStream_t s, cudaEvent_t e) { return cudaStreamWaitEvent(s, e, 0); }
inline cudaError_t graph_begin(cudaStream_t s) { return cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal); }
inline cudaError_t graph_end(cudaStream_t s, cudaGraphExec_t *exec)
{
    cudaGraph_t g = nullptr;
    cudaError_t r = cudaStreamEndCapture(s, &g);
    if (r != cudaSuccess)
        return r;
    r = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    return r;
}
inline cudaError_t graph_launch(cudaGraphExec_t e, cudaStream_t s) { return cudaGraphLaunch(e, s); }
inline void graph_free(cudaGraphExec_t e)
{
    if (e)
        cudaGraphExecDestroy(e);
}
} // namespace dndsb
