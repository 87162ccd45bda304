// FP32 and FP64 fused multiply-add throughput of this GPU, for the ALU
// roofline the benchmark reports beside the HBM one: every thread runs
// independent FMA chains in registers (no memory traffic but one store).
#include "common.cuh"

namespace {

template <typename R>
__global__ void __launch_bounds__(256) fma_probe_kernel(R *out, int iters, R a, R b)
{
    R x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = (R)(threadIdx.x + k) * (R)1e-3;
    for (int i = 0; i < iters; i++)
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
    R s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == (R)12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" {

// Measured FMA throughput in GFLOP/s (2 flops per FMA) for FP32 (fp64 = 0)
// or FP64 (fp64 = 1), from `reps` launches of a fixed-size probe.
int pinyb200_fma_peak(int fp64, int reps, double *gflops)
{
    if (!gflops || reps < 1) return pinyb200::record_error(nullptr, PINYB200_ERR_ARG, "fma_peak: bad arguments");
    int dev = 0, sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return pinyb200::record_error(nullptr, PINYB200_ERR_NO_DEVICE, "fma_peak: no device");
    const int blocks = sm * 8, threads = 256, iters = 4096;
    void *out = nullptr;
    if (cudaMalloc(&out, (size_t)blocks * threads * 8) != cudaSuccess)
        return pinyb200::record_error(nullptr, PINYB200_ERR_CUDA, "fma_peak: allocation failed");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int r = 0; r <= reps; r++) {
        cudaEventRecord(e0);
        if (fp64) fma_probe_kernel<double><<<blocks, threads>>>((double *)out, iters, 0.999999, 1e-7);
        else fma_probe_kernel<float><<<blocks, threads>>>((float *)out, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return pinyb200::record_error(nullptr, PINYB200_ERR_CUDA, cudaGetErrorString(err));
    *gflops = 2.0 * 8.0 * (double)iters * blocks * threads / (best * 1e-3) / 1e9;
    return PINYB200_OK;
}

}  // extern "C"
