// calib.cu -- measured FP64 / FP32 FMA throughput of the current device.
//
// The Euler kernels are bound by the FP64 (or FP32) pipe, not by HBM; this
// kernel measures that pipe's sustained rate (independent FMA chains, all SMs
// busy) so the benchmark can report a roofline fraction against a measured
// number rather than a datasheet figure.
#include "cn_internal.h"

namespace cn {

template <typename T>
__global__ void __launch_bounds__(256) fma_chains(T *out, int iters, T a, T b)
{
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = T(threadIdx.x + k) * T(1e-3);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == T(12345.678)) out[0] = s; // keeps the chains alive
}

template <typename T> static cn_status run(double *tflops)
{
    int sms = 0, dev = 0;
    CN_CUDA_TRY(cudaGetDevice(&dev));
    CN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    T *out = nullptr;
    CN_CUDA_TRY(cudaMalloc(&out, sizeof(T)));
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_chains<T><<<blocks, threads>>>(out, 256, T(0.999), T(1e-4)); // warm-up
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(e0);
        fma_chains<T><<<blocks, threads>>>(out, iters, T(0.999), T(1e-4));
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        best = ms < best ? ms : best;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess) return cuda_fail(err, "fma_chains");
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return CN_OK;
}

} // namespace cn

extern "C" cn_status cn_calib_fma_peak(cn_dtype dtype, double *tflops)
{
    if (!tflops) return cn::fail(CN_ERR_INVALID_ARGUMENT, "tflops is NULL");
    if (dtype == CN_FLOAT64) return cn::run<double>(tflops);
    if (dtype == CN_FLOAT32) return cn::run<float>(tflops);
    return cn::fail(CN_ERR_UNSUPPORTED, "dtype must be FLOAT32 or FLOAT64");
}
