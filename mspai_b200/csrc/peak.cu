// CUDA-core FMA throughput probe: the roofline denominator of the FP32 / FP64
// least-squares kernels (tensor cores are not used by this library).
#include "mspai_b200.h"

#include <cuda_runtime.h>

namespace {

template <class T>
__global__ void __launch_bounds__(256) fma_chain_kernel(T* out, int iters, T a, T b)
{
    // 8 independent chains per thread keep the FMA pipes full
    T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5,
      x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            x0 = fma(x0, a, b);
            x1 = fma(x1, a, b);
            x2 = fma(x2, a, b);
            x3 = fma(x3, a, b);
            x4 = fma(x4, a, b);
            x5 = fma(x5, a, b);
            x6 = fma(x6, a, b);
            x7 = fma(x7, a, b);
        }
    }
    const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == T(-1234.5))  // never true; keeps the chains alive
        out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <class T>
int run(int device, double* gflops)
{
    if (cudaSetDevice(device) != cudaSuccess)
        return MSPAI_ERR_NO_DEVICE;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256, iters = 2048;
    T* out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * blocks * threads) != cudaSuccess)
        return MSPAI_ERR_ALLOC;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_chain_kernel<T><<<blocks, threads>>>(out, iters / 8, T(0.999), T(0.001));  // warm-up
    cudaEventRecord(e0);
    fma_chain_kernel<T><<<blocks, threads>>>(out, iters, T(0.999), T(0.001));
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess || ms <= 0.f)
        return MSPAI_ERR_CUDA;
    const double flops = 2.0 * 8.0 * 16.0 * iters * static_cast<double>(blocks) * threads;
    *gflops = flops / (ms * 1e-3) * 1e-9;
    return MSPAI_OK;
}

}  // namespace

extern "C" int mspai_measure_fma_peak(int32_t device, int32_t fp64, double* gflops)
{
    if (!gflops)
        return MSPAI_ERR_PARAM;
    return fp64 ? run<double>(device, gflops) : run<float>(device, gflops);
}
