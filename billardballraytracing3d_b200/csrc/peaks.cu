// Pipe-peak microbenchmarks for the roofline denominators the driver does
// not measure: FP64 and FP32 FMA throughput and L2-resident read bandwidth.
// Each kernel runs a fixed, bounded amount of work; timing is by CUDA events.
#include <cuda_runtime.h>

#include "../../include/bbrt.h"

namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_chain(T* out, int iters, T a, T b) {
    // 8 independent FMA chains per thread hide the pipe latency.
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = static_cast<T>(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == static_cast<T>(-1.2345)) out[threadIdx.x] = s;   // keeps the chains live
}

__global__ void __launch_bounds__(256) k_read(const float4* __restrict__ buf, size_t n4, int reps, float* out) {
    float acc = 0.0f;
    for (int r = 0; r < reps; ++r) {
        for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n4;
             i += static_cast<size_t>(gridDim.x) * blockDim.x) {
            const float4 v = __ldcg(buf + i);
            acc += v.x + v.y + v.z + v.w;
        }
    }
    if (acc == -1.0f) out[0] = acc;
}

int sms() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

template <typename T>
int fma_peak(double* tflops) {
    T* out = nullptr;
    if (cudaMalloc(&out, 256 * sizeof(T)) != cudaSuccess) return BBRT_ERR_CUDA;
    const int blocks = sms() * 8, iters = 1 << 14;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_chain<T><<<blocks, 256>>>(out, 64, static_cast<T>(0.999), static_cast<T>(0.001));
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0);
        k_fma_chain<T><<<blocks, 256>>>(out, iters, static_cast<T>(0.999), static_cast<T>(0.001));
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return BBRT_ERR_CUDA;
    const double flop = 2.0 * 8.0 * iters * static_cast<double>(blocks) * 256.0;
    *tflops = flop / (best * 1e-3) / 1e12;
    return BBRT_OK;
}

int l2_read_peak(double* gbs) {
    const size_t bytes = 48ull << 20;   // resident in the 126 MB L2
    float4* buf = nullptr;
    float* out = nullptr;
    if (cudaMalloc(&buf, bytes) != cudaSuccess) return BBRT_ERR_CUDA;
    if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) { cudaFree(buf); return BBRT_ERR_CUDA; }
    cudaMemset(buf, 0, bytes);
    const size_t n4 = bytes / sizeof(float4);
    const int blocks = sms() * 8, reps = 20;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_read<<<blocks, 256>>>(buf, n4, 1, out);
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0);
        k_read<<<blocks, 256>>>(buf, n4, reps, out);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    cudaFree(out);
    if (err != cudaSuccess) return BBRT_ERR_CUDA;
    *gbs = static_cast<double>(bytes) * reps / (best * 1e-3) / 1e9;
    return BBRT_OK;
}

}  // namespace

extern "C" BBRT_API int bbrt_measure_pipe_peak(int pipe, double* value) {
    if (!value) return BBRT_ERR_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return BBRT_ERR_CUDA;
    switch (pipe) {
        case BBRT_PIPE_FP64: return fma_peak<double>(value);
        case BBRT_PIPE_FP32: return fma_peak<float>(value);
        case BBRT_PIPE_L2: return l2_read_peak(value);
        default: return BBRT_ERR_ARG;
    }
}
