// FP64 throughput probes: the denominators of the compute roofline of H·psi (the
// kinetic kernel runs on the FP64 tensor pipe, the mixing kernel on the FP64 FMA pipe).
// Each thread (warp) runs 8 independent accumulation chains so that the pipe, not the
// dependency latency, sets the rate; the result is written only if it is impossible,
// which keeps the chains live without memory traffic.
#include "common.cuh"
#include "operator.cuh"

namespace {

__device__ __forceinline__ void peak_dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void dmma_peak_kernel(double *sink, int iters)
{
    double acc[8][2] = {};
    const double a = 1.0 + 1e-12 * threadIdx.x, b = 1.0 - 1e-12 * threadIdx.x;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) peak_dmma(acc[q][0], acc[q][1], a, b);
    }
    double s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += acc[q][0] + acc[q][1];
    if (s == -1.0) sink[threadIdx.x] = s;
}

__global__ void dfma_peak_kernel(double *sink, int iters)
{
    double acc[8] = {};
    const double a = 1.0 + 1e-12 * threadIdx.x, b = 1e-9;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] = fma(a, acc[q], b);
    }
    double s = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += acc[q];
    if (s == -1.0) sink[threadIdx.x] = s;
}

}  // namespace

extern "C" int he_fp64_peak(int kind, int iters, double *tflops, void *stream)
{
    if (!tflops || iters < 1 || (kind != 0 && kind != 1)) return he_fail(HE_ERR_ARG, "bad probe arguments", __FILE__, __LINE__);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    int device = 0, sms = 0;
    HE_CUDA_TRY(cudaGetDevice(&device));
    HE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int blocks = 4 * sms, threads = 256;
    double *sink = nullptr;
    HE_CUDA_TRY(cudaMalloc(&sink, threads * sizeof(double)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float ms = 0;
    if (e == cudaSuccess) {
        for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {   // the first launch warms the clocks up
            e = cudaEventRecord(e0, s);
            if (kind == 0) dmma_peak_kernel<<<blocks, threads, 0, s>>>(sink, iters);
            else dfma_peak_kernel<<<blocks, threads, 0, s>>>(sink, iters);
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaEventRecord(e1, s);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        }
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) { he_set_error(cudaGetErrorString(e), __FILE__, __LINE__); return HE_ERR_CUDA; }
    // DMMA m8n8k4: 8 x 8 x 4 FMAs per warp instruction; DFMA: one FMA per thread
    const double flops = kind == 0 ? (double)blocks * (threads / 32) * iters * 8 * (8 * 8 * 4 * 2)
                                   : (double)blocks * threads * iters * 8 * 2;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return HE_OK;
}
