// Shared device/host helpers for the B200 helium propagation engine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/helium_b200.h"

// ---------------------------------------------------------------------------------
// Complex arithmetic on interleaved (re, im) pairs.  double2 / float2 give 16 / 8 B
// aligned vector loads; every routine is written as explicit FMAs.
// ---------------------------------------------------------------------------------
template <typename R> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float> { using type = float2; };
template <typename R> using cplx = typename cplx_t<R>::type;

template <typename R> __host__ __device__ __forceinline__ cplx<R> mk(R re, R im) { cplx<R> z; z.x = re; z.y = im; return z; }
template <typename R> __host__ __device__ __forceinline__ cplx<R> cadd(cplx<R> a, cplx<R> b) { return mk<R>(a.x + b.x, a.y + b.y); }
template <typename R> __host__ __device__ __forceinline__ cplx<R> csub(cplx<R> a, cplx<R> b) { return mk<R>(a.x - b.x, a.y - b.y); }
template <typename R> __host__ __device__ __forceinline__ cplx<R> cmul(cplx<R> a, cplx<R> b) {
    return mk<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// acc + a*b
template <typename R> __host__ __device__ __forceinline__ cplx<R> cfma(cplx<R> a, cplx<R> b, cplx<R> acc) {
    acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
// acc + s*b for real s
template <typename R> __host__ __device__ __forceinline__ cplx<R> rfma(R s, cplx<R> b, cplx<R> acc) {
    acc.x = fma(s, b.x, acc.x); acc.y = fma(s, b.y, acc.y); return acc;
}
// conj(a)*b accumulated
template <typename R> __host__ __device__ __forceinline__ cplx<R> cfma_conj(cplx<R> a, cplx<R> b, cplx<R> acc) {
    acc.x = fma(a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
template <typename R> __host__ __device__ __forceinline__ cplx<R> cscale(R s, cplx<R> a) { return mk<R>(s * a.x, s * a.y); }
template <typename R> __host__ __device__ __forceinline__ R cabs2(cplx<R> a) { return a.x * a.x + a.y * a.y; }

template <typename R> __device__ __forceinline__ cplx<R> ldg(const cplx<R>* p) { return __ldg(p); }

// ---------------------------------------------------------------------------------
// Sum of nb per-block partials p[b * stride] by one warp in a fixed order: lane l adds
// b = l, l + 32, ... in sequence, then a butterfly over the lanes.  Every lane returns
// the same value and the order never depends on timing, so results are reproducible.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ double warp_fixed_sum(const double* p, int nb, size_t stride)
{
    const int lane = threadIdx.x & 31;
    double s = 0;
    for (int b = lane; b < nb; b += 32) s += p[(size_t)b * stride];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    return s;
}

__device__ __forceinline__ double2 warp_fixed_sum(const double2* p, int nb, size_t stride)
{
    const int lane = threadIdx.x & 31;
    double2 s = mk<double>(0, 0);
    for (int b = lane; b < nb; b += 32) s = cadd<double>(s, p[(size_t)b * stride]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, off);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, off);
    }
    return s;
}

// ---------------------------------------------------------------------------------
// Device-resident operator tables.  Indices are zero based, psi(i,j,c) has i fastest
// (the reference's Fortran order, src/kernels.f90:125).
// ---------------------------------------------------------------------------------
namespace he {
// Fields of a batch of instances that share one operator (passed by value to kernels):
// instance b of a batched apply sees the field f[b][0..2]; a single apply has count 1.
// skip (optional): a device flag that, when non-zero at launch, makes the banded kinetic and
// generated mixing kernels (the default path) return without work (the done word of a Krylov
// solve, so the applies a fused solve enqueues past its convergence cost one empty launch
// each).  The other kernel paths (he_set_path 0, 2, 3; he_set_mix 0) ignore it: there those
// applies run in full and their results are discarded.
constexpr int HE_BATCH_MAX = 64;
struct FieldBatch {
    int count;
    double f[HE_BATCH_MAX][3];
    const int *skip;
};

template <typename R> struct DeviceTables {
    int n, nc, nt, nv, nd, nlam;
    int diag_separable;                 // 1: diag(i,j,c) = d1(i,c) + d2(j,c)
    const int* ptr; const int* col; const cplx<R>* tv;
    const cplx<R>* diag;                // n*n*nc when !diag_separable
    const cplx<R>* d1; const cplx<R>* d2;   // n*nc each when diag_separable
    const int* vptr; const int* vc; const int* vl; const cplx<R>* vcoef;
    const cplx<R>* rad;                 // n*n*nlam
    const int* dptr; const int* dc; const int* de; const cplx<R>* dcoef; const R* ldiff;
    const cplx<R>* r;
    const cplx<R>* hinv;                // 1/(2 r), n entries
};
}  // namespace he

#define HE_CUDA_TRY(expr)                                                                     \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess) { he_set_error(cudaGetErrorString(_e), __FILE__, __LINE__); return HE_ERR_CUDA; } \
    } while (0)

void he_set_error(const char* what, const char* file, int line);

// Looks up (and under lazy module loading, loads) the allocation-free entry point's static
// scratch on the current device (noalloc.cu).
int he_noalloc_prepare_device();

// Raise a kernel's dynamic shared-memory limit on the current device, once per kernel,
// device and size (the attribute call costs microseconds per launch otherwise).
cudaError_t he_smem_limit(const void* kernel, size_t bytes);
