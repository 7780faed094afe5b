// Separable ionic resolvent preconditioner (python/implicit.py:13-39) on the device.
//
// For channel c with one-electron angular momenta (l1, l2) and the eigendecompositions
// H_l = S_l diag(e_l) S_l^-1 of the ionic radial Hamiltonians (computed on the host):
//   Z_c = S_{l1}^-1 Psi_c (S_{l2}^-1)^T,   Z_c(i,j) /= 1 + i alpha (e_{l1}(i) + e_{l2}(j) + shift),
//   Y_c = S_{l1} Z_c S_{l2}^T
// with Psi_c the n x n column-major slice psi(:, :, c) (the reference's u[c] is its
// transpose, so I2 u I1^T there is I1 Psi I2^T here).  The four n^3 products per channel
// are plain batched GEMMs and run in cuBLAS (complex128: ZGEMM, complex64: CGEMM); the
// scaling and the precision conversions are this file's kernels.
#include <cublas_v2.h>

#include <vector>

#include "common.cuh"
#include "operator.cuh"

struct he_separable {
    int device = 0, n = 0, nc = 0, nl = 0, precision = 0;
    cublasHandle_t blas = nullptr;
    void *S = nullptr, *I = nullptr;      // nl matrices each (n x n, column major)
    void *evals = nullptr;                // nl x n
    int *l1 = nullptr, *l2 = nullptr;     // per channel (device)
    void *buf[2] = {nullptr, nullptr};    // two n*n*nc work vectors of the precision
    void **ptrs = nullptr;                // 3 x nc device pointer arrays
    ~he_separable()
    {
        if (blas) cublasDestroy(blas);
        cudaFree(S); cudaFree(I); cudaFree(evals); cudaFree(l1); cudaFree(l2);
        cudaFree(buf[0]); cudaFree(buf[1]); cudaFree(ptrs);
    }
};

namespace he {

template <typename R>
__global__ void fill_ptrs_kernel(int nc, size_t nn, const cplx<R> *mats, const int *lsel, const cplx<R> *bbase,
                                 cplx<R> *cbase, int mode, void **ptrs)
{
    // mode 0: A = mats[lsel[c]], B = bbase + c nn, C = cbase + c nn
    // mode 1: A = bbase + c nn,  B = mats[lsel[c]], C = cbase + c nn
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const cplx<R> *m = mats + (size_t)lsel[c] * nn;
        const cplx<R> *v = bbase + (size_t)c * nn;
        ptrs[c] = (void *)(mode == 0 ? m : v);
        ptrs[nc + c] = (void *)(mode == 0 ? v : m);
        ptrs[2 * nc + c] = (void *)(cbase + (size_t)c * nn);
    }
}

template <typename R>
__global__ void resolvent_scale_kernel(int n, int nc, const cplx<R> *__restrict__ evals, const int *__restrict__ l1,
                                       const int *__restrict__ l2, cplx<R> alpha, R shift, cplx<R> *z)
{
    const size_t nn = (size_t)n * n, total = nn * nc;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(p / nn);
        const size_t q = p % nn;
        const int i = (int)(q % n), j = (int)(q / n);
        const cplx<R> e = cadd<R>(evals[(size_t)l1[c] * n + i], evals[(size_t)l2[c] * n + j]);
        const cplx<R> es = mk<R>(e.x + shift, e.y);
        const cplx<R> ia = mk<R>(-alpha.y, alpha.x);
        const cplx<R> den = cfma<R>(ia, es, mk<R>(1, 0));
        const R d2 = cabs2<R>(den);
        const cplx<R> v = z[p];
        z[p] = mk<R>((v.x * den.x + v.y * den.y) / d2, (v.y * den.x - v.x * den.y) / d2);
    }
}

__global__ void to_c64_kernel(size_t n, const double2 *x, float2 *y)
{
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        y[p] = make_float2((float)x[p].x, (float)x[p].y);
}

__global__ void to_c128_kernel(size_t n, const float2 *x, double2 *y)
{
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        y[p] = make_double2((double)x[p].x, (double)x[p].y);
}

static int gemm_batched(he_separable *h, bool transb, void **ptrs)
{
    const int n = h->n;
    cublasStatus_t st;
    if (h->precision == HE_C128) {
        const cuDoubleComplex one = make_cuDoubleComplex(1, 0), zero = make_cuDoubleComplex(0, 0);
        st = cublasZgemmBatched(h->blas, CUBLAS_OP_N, transb ? CUBLAS_OP_T : CUBLAS_OP_N, n, n, n, &one,
                                (const cuDoubleComplex **)ptrs, n, (const cuDoubleComplex **)(ptrs + h->nc), n, &zero,
                                (cuDoubleComplex **)(ptrs + 2 * h->nc), n, h->nc);
    } else {
        const cuComplex one = make_cuComplex(1, 0), zero = make_cuComplex(0, 0);
        st = cublasCgemmBatched(h->blas, CUBLAS_OP_N, transb ? CUBLAS_OP_T : CUBLAS_OP_N, n, n, n, &one,
                                (const cuComplex **)ptrs, n, (const cuComplex **)(ptrs + h->nc), n, &zero,
                                (cuComplex **)(ptrs + 2 * h->nc), n, h->nc);
    }
    if (st != CUBLAS_STATUS_SUCCESS) return he_fail(HE_ERR_CUDA, "cuBLAS batched GEMM failed", __FILE__, __LINE__);
    return HE_OK;
}

template <typename R>
static int apply_t(he_separable *h, const cplx<R> *src, cplx<R> *dst, double2 alpha, double shift, cudaStream_t s)
{
    const size_t nn = (size_t)h->n * h->n;
    const cplx<R> *S = static_cast<const cplx<R> *>(h->S), *I = static_cast<const cplx<R> *>(h->I);
    cplx<R> *b0 = static_cast<cplx<R> *>(h->buf[0]), *b1 = static_cast<cplx<R> *>(h->buf[1]);
    int rc;
    // b1 = I_{l1} Psi ; b0 = b1 I_{l2}^T
    fill_ptrs_kernel<R><<<1, 256, 0, s>>>(h->nc, nn, I, h->l1, src, b1, 0, h->ptrs);
    if ((rc = gemm_batched(h, false, h->ptrs))) return rc;
    fill_ptrs_kernel<R><<<1, 256, 0, s>>>(h->nc, nn, I, h->l2, b1, b0, 1, h->ptrs);
    if ((rc = gemm_batched(h, true, h->ptrs))) return rc;
    resolvent_scale_kernel<R><<<592, 256, 0, s>>>(h->n, h->nc, static_cast<const cplx<R> *>(h->evals), h->l1, h->l2,
                                                  mk<R>((R)alpha.x, (R)alpha.y), (R)shift, b0);
    // b1 = S_{l1} Z ; dst = b1 S_{l2}^T
    fill_ptrs_kernel<R><<<1, 256, 0, s>>>(h->nc, nn, S, h->l1, b0, b1, 0, h->ptrs);
    if ((rc = gemm_batched(h, false, h->ptrs))) return rc;
    fill_ptrs_kernel<R><<<1, 256, 0, s>>>(h->nc, nn, S, h->l2, b1, dst, 1, h->ptrs);
    if ((rc = gemm_batched(h, true, h->ptrs))) return rc;
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

}  // namespace he

using namespace he;

extern "C" int he_separable_create(he_separable **out, int n, int nc, int nl, const double *S, const double *Sinv,
                                   const double *evals, const int *l1, const int *l2, int precision)
{
    if (!out || !S || !Sinv || !evals || !l1 || !l2 || n < 1 || nc < 1 || nl < 1)
        return he_fail(HE_ERR_ARG, "bad separable preconditioner argument", __FILE__, __LINE__);
    if (precision != HE_C128 && precision != HE_C64) return he_fail(HE_ERR_ARG, "bad precision", __FILE__, __LINE__);
    for (int c = 0; c < nc; ++c)
        if (l1[c] < 0 || l1[c] >= nl || l2[c] < 0 || l2[c] >= nl)
            return he_fail(HE_ERR_SHAPE, "channel angular momentum outside the eigenbasis table", __FILE__, __LINE__);
    *out = nullptr;
    he_separable *h = new he_separable();
    h->n = n; h->nc = nc; h->nl = nl; h->precision = precision;
    const size_t nn = (size_t)n * n, elem = precision == HE_C128 ? sizeof(double2) : sizeof(float2);
    auto fail = [&](cudaError_t e) { he_set_error(cudaGetErrorString(e), __FILE__, __LINE__); delete h; return HE_ERR_CUDA; };
    cudaError_t e = cudaGetDevice(&h->device);
    auto put = [&](void **dst, const double *src, size_t count) -> cudaError_t {
        cudaError_t r = cudaMalloc(dst, count * elem);
        if (r != cudaSuccess) return r;
        if (precision == HE_C128) return cudaMemcpy(*dst, src, count * elem, cudaMemcpyHostToDevice);
        std::vector<float2> tmp(count);
        for (size_t k = 0; k < count; ++k) tmp[k] = make_float2((float)src[2 * k], (float)src[2 * k + 1]);
        return cudaMemcpy(*dst, tmp.data(), count * elem, cudaMemcpyHostToDevice);
    };
    if (e == cudaSuccess) e = put(&h->S, S, nl * nn);
    if (e == cudaSuccess) e = put(&h->I, Sinv, nl * nn);
    if (e == cudaSuccess) e = put(&h->evals, evals, (size_t)nl * n);
    if (e == cudaSuccess) e = cudaMalloc(&h->l1, nc * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(h->l1, l1, nc * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&h->l2, nc * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(h->l2, l2, nc * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&h->buf[0], nn * nc * elem);
    if (e == cudaSuccess) e = cudaMalloc(&h->buf[1], nn * nc * elem);
    if (e == cudaSuccess) e = cudaMalloc(&h->ptrs, 3 * (size_t)nc * sizeof(void *));
    if (e != cudaSuccess) return fail(e);
    if (cublasCreate(&h->blas) != CUBLAS_STATUS_SUCCESS) {
        delete h;
        return he_fail(HE_ERR_CUDA, "cublasCreate failed", __FILE__, __LINE__);
    }
    *out = h;
    return HE_OK;
}

extern "C" int he_separable_destroy(he_separable *h)
{
    delete h;
    return HE_OK;
}

// y = M(alpha, shift) x ; x, y complex128 device vectors of n*n*nc elements (y != x).
extern "C" int he_separable_apply(he_separable *h, const void *x, void *y, double alpha_re, double alpha_im,
                                  double shift, void *stream)
{
    if (!h || !x || !y || x == y) return he_fail(HE_ERR_ARG, "bad separable apply argument", __FILE__, __LINE__);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cublasSetStream(h->blas, s) != CUBLAS_STATUS_SUCCESS)
        return he_fail(HE_ERR_CUDA, "cublasSetStream failed", __FILE__, __LINE__);
    const double2 alpha = mk<double>(alpha_re, alpha_im);
    const size_t total = (size_t)h->n * h->n * h->nc;
    if (h->precision == HE_C128)
        return apply_t<double>(h, static_cast<const double2 *>(x), static_cast<double2 *>(y), alpha, shift, s);
    // complex64: convert in, work in the buffers, convert out (python/implicit.py:35-39 .to(dtype)).
    // buf[0] holds the input; the GEMMs alternate buf[0] -> buf[1] -> buf[0] -> buf[1] -> buf[0],
    // so no product reads and writes the same buffer.
    float2 *b0 = static_cast<float2 *>(h->buf[0]);
    to_c64_kernel<<<592, 256, 0, s>>>(total, static_cast<const double2 *>(x), b0);
    int rc = apply_t<float>(h, b0, b0, alpha, shift, s);
    if (rc) return rc;
    to_c128_kernel<<<592, 256, 0, s>>>(total, b0, static_cast<double2 *>(y));
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}
