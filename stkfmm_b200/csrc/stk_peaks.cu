// stk_peaks.cu -- CUDA-core throughput probes for the P2P roofline.
//
// The P2P kernels are bound by the FP32 pipe (mixed path), the FP64 pipe (plain
// path) and the MUFU/XU unit (rsqrt), none of which the HBM / tensor-core peak
// figures describe.  These kernels measure, on the running GPU: FP32 FMA/s,
// FP64 FMA/s and MUFU rsqrt/s, each with independent dependency chains so the
// pipe (not latency) is the limit, plus the effective SM clock seen meanwhile.
#include <cuda_runtime.h>

#include "../../include/stkfmm_b200.h"

namespace {

constexpr int kChains = 8;

__global__ void fp32_fma_kernel(float *out, int iters, float a, float b) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = threadIdx.x * 1e-7f + c;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) x[c] = fmaf(x[c], a, b);
    }
    float s = 0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += x[c];
    if (s == 1234.5f) out[threadIdx.x] = s;  // never true: keeps the chains alive
}

__global__ void fp64_fma_kernel(double *out, int iters, double a, double b) {
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = threadIdx.x * 1e-7 + c;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) x[c] = fma(x[c], a, b);
    }
    double s = 0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += x[c];
    if (s == 1234.5) out[threadIdx.x] = s;
}

__global__ void fp32x2_fma_kernel(float *out, int iters, float a, float b) {
    float2 x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = make_float2(threadIdx.x * 1e-7f + c, c + 0.5f);
    const float2 av = make_float2(a, a), bv = make_float2(b, b);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) x[c] = __ffma2_rn(x[c], av, bv);
    }
    float s = 0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += x[c].x + x[c].y;
    if (s == 1234.5f) out[threadIdx.x] = s;
}

__global__ void mufu_rsqrt_kernel(float *out, int iters) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = 1.0f + threadIdx.x * 1e-6f + c;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) {
            float y;
            asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x[c]));
            x[c] = y;
        }
    }
    float s = 0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += x[c];
    if (s == 1234.5f) out[threadIdx.x] = s;
}

__global__ void clock_kernel(long long *out, long long spin) {
    long long c0 = clock64();
    unsigned long long t0, t1;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    while (clock64() - c0 < spin) {
    }
    long long c1 = clock64();
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
    out[0] = c1 - c0;
    out[1] = (long long)(t1 - t0);
}

template <class F>
float time_ms(F launch, cudaStream_t s) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch();  // warm-up
    cudaEventRecord(e0, s);
    launch();
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms;
}

}  // namespace

// out[0] FP32 TFLOP/s (FMA = 2), out[1] FP64 TFLOP/s, out[2] MUFU rsqrt Gop/s,
// out[3] SM clock in MHz measured by clock64 / globaltimer, out[4] SM count,
// out[5] packed FP32 (fma.rn.f32x2) TFLOP/s.
extern "C" int stk_measure_peaks(double *out) {
    if (!out) return STK_ERR_INVALID_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return STK_ERR_NO_DEVICE;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float *fbuf = nullptr;
    long long *cbuf = nullptr;
    if (cudaMalloc(&fbuf, 1024 * sizeof(double)) != cudaSuccess) return STK_ERR_CUDA;
    if (cudaMalloc(&cbuf, 2 * sizeof(long long)) != cudaSuccess) {
        cudaFree(fbuf);
        return STK_ERR_CUDA;
    }
    cudaStream_t s = 0;
    const int threads = 256, blocks = sms * 8;
    const double nthr = (double)threads * blocks;
    const int it32 = 4096, it64 = 2048, itmu = 1024;
    float ms = time_ms([&] { fp32_fma_kernel<<<blocks, threads, 0, s>>>(fbuf, it32, 0.999f, 1e-3f); }, s);
    out[0] = nthr * it32 * kChains * 2.0 / (ms * 1e-3) / 1e12;
    ms = time_ms([&] { fp64_fma_kernel<<<blocks, threads, 0, s>>>((double *)fbuf, it64, 0.999, 1e-3); }, s);
    out[1] = nthr * it64 * kChains * 2.0 / (ms * 1e-3) / 1e12;
    ms = time_ms([&] { mufu_rsqrt_kernel<<<blocks, threads, 0, s>>>(fbuf, itmu); }, s);
    out[2] = nthr * itmu * kChains / (ms * 1e-3) / 1e9;
    ms = time_ms([&] { fp32x2_fma_kernel<<<blocks, threads, 0, s>>>(fbuf, it32 / 2, 0.999f, 1e-3f); }, s);
    out[5] = nthr * (it32 / 2) * kChains * 4.0 / (ms * 1e-3) / 1e12;
    clock_kernel<<<1, 1, 0, s>>>(cbuf, 20000000LL);
    long long h[2] = {0, 1};
    cudaMemcpy(h, cbuf, sizeof(h), cudaMemcpyDeviceToHost);
    out[3] = h[1] > 0 ? (double)h[0] / (double)h[1] * 1e3 : 0.0;
    out[4] = sms;
    cudaError_t err = cudaGetLastError();
    cudaFree(fbuf);
    cudaFree(cbuf);
    return err == cudaSuccess ? STK_OK : STK_ERR_CUDA;
}
