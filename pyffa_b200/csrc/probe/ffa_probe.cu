// ffa_probe.cu -- measurement helper for the benchmark's roofline (not part
// of the tracking ABI): float64 and float32 FMA throughput kernels giving the
// FP64 and FP32 pipe peaks of the device they run on.
#include <cuda_runtime.h>
#include <stdint.h>

__global__ void __launch_bounds__(256) fp64_fma_kernel(double *out, int iters, double a, double b)
{
    double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-3, x2 = x0 + 2e-3, x3 = x0 + 3e-3;
    double x4 = x0 + 4e-3, x5 = x0 + 5e-3, x6 = x0 + 6e-3, x7 = x0 + 7e-3;
    for (int i = 0; i < iters; ++i) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 12345.678) out[blockIdx.x] = s;  // keeps the loop live
}

extern "C" int ffa_probe_fp64_fma(int blocks, int iters, double *out, void *stream, float *ms)
{
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fp64_fma_kernel<<<blocks, 256, 0, s>>>(out, iters, 0.999999, 1e-7);  // warm-up
    cudaEventRecord(e0, s);
    fp64_fma_kernel<<<blocks, 256, 0, s>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

__global__ void __launch_bounds__(256) fp32_fma_kernel(float *out, int iters, float a, float b)
{
    float x0 = threadIdx.x * 1e-9f, x1 = x0 + 1e-3f, x2 = x0 + 2e-3f, x3 = x0 + 3e-3f;
    float x4 = x0 + 4e-3f, x5 = x0 + 5e-3f, x6 = x0 + 6e-3f, x7 = x0 + 7e-3f;
    for (int i = 0; i < iters; ++i) {
        x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
        x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
    }
    float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the loop live
}

extern "C" int ffa_probe_fp32_fma(int blocks, int iters, float *out, void *stream, float *ms)
{
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fp32_fma_kernel<<<blocks, 256, 0, s>>>(out, iters, 0.999999f, 1e-7f);  // warm-up
    cudaEventRecord(e0, s);
    fp32_fma_kernel<<<blocks, 256, 0, s>>>(out, iters, 0.999999f, 1e-7f);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
