// He+ (ionic) operator for the backward propagation of the tSURFF channel functions
// chi_c(t): a sparse matrix with a handful of coefficient planes,
//   H(c) = sum_k c_k M_k   (M_0 = H0^dagger, M_1..3 = P_a^dagger, M_4 = identity; the reference's
//   IonicAdjoint operator, python/ionic_adjoint.py:16-21, 41-50),
// applied to nrhs right-hand sides at once (x[row][rhs], row-major), plus the exact
// per-angular-block resolvent of H0^dagger used as the GMRES preconditioner
// (python/ionic_adjoint.py:24-39).  The CF4 / Pade / GMRES driver above is shared with the
// two-electron propagation.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "operator.cuh"

struct he_ionic {
    int device = 0;
    int ndof = 0, nrhs = 0, nmat = 0;
    long long nnz = 0;
    int *ptr = nullptr, *col = nullptr;
    double2 *data = nullptr;                 // nmat planes of nnz values
    int na = 0, n = 0;                       // preconditioner blocks
    double2 *S = nullptr, *Si = nullptr, *E = nullptr;   // na x (n x n column major), na x n
    ~he_ionic()
    {
        cudaFree(ptr); cudaFree(col); cudaFree(data); cudaFree(S); cudaFree(Si); cudaFree(E);
    }
};

namespace {

constexpr int IONIC_MAX_MATS = 16;
constexpr int IONIC_MAX_RHS = 16;
struct Coefs {
    double c[IONIC_MAX_MATS];
};

// One warp per row: lanes take the row's non-zeros in turn, accumulate every right-hand
// side, then a fixed-order butterfly.  shifted: y = x + i alpha (H x - shift x); else y = H x.
__global__ void ionic_apply_kernel(int ndof, int nrhs, int nmat, long long nnz, const int *__restrict__ ptr,
                                   const int *__restrict__ col, const double2 *__restrict__ data, Coefs cf,
                                   const double2 *__restrict__ x, double2 *__restrict__ y, double2 alpha, double shift,
                                   int shifted)
{
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= ndof) return;
    double2 acc[IONIC_MAX_RHS];
#pragma unroll
    for (int r = 0; r < IONIC_MAX_RHS; ++r) acc[r] = mk<double>(0, 0);
    for (int e = ptr[row] + lane; e < ptr[row + 1]; e += 32) {
        double2 v = mk<double>(0, 0);
        for (int k = 0; k < nmat; ++k) v = rfma<double>(cf.c[k], data[(size_t)k * nnz + e], v);
        const double2 *xr = x + (size_t)col[e] * nrhs;
#pragma unroll
        for (int r = 0; r < IONIC_MAX_RHS; ++r)
            if (r < nrhs) acc[r] = cfma<double>(v, xr[r], acc[r]);
    }
#pragma unroll
    for (int r = 0; r < IONIC_MAX_RHS; ++r) {
        if (r >= nrhs) break;
        double2 s = acc[r];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            s.x += __shfl_xor_sync(0xffffffffu, s.x, off);
            s.y += __shfl_xor_sync(0xffffffffu, s.y, off);
        }
        if (lane == r) {
            const size_t i = (size_t)row * nrhs + r;
            if (shifted) {
                const double2 xi = x[i];
                const double2 t = mk<double>(s.x - shift * xi.x, s.y - shift * xi.y);   // H x - shift x
                const double2 ia = mk<double>(-alpha.y, alpha.x);                         // i alpha
                y[i] = cfma<double>(ia, t, xi);
            } else {
                y[i] = s;
            }
        }
    }
}

// y_a = S_a [ (Si_a x_a) / (1 + i alpha (E_a + shift)) ] for block a = blockIdx.x and
// right-hand side r = blockIdx.y; x_a is rows a n .. a n + n - 1 of column r.
__global__ void ionic_precondition_kernel(int n, int nrhs, const double2 *__restrict__ S, const double2 *__restrict__ Si,
                                          const double2 *__restrict__ E, const double2 *__restrict__ x,
                                          double2 *__restrict__ y, double2 alpha, double shift)
{
    extern __shared__ double2 buf[];   // 2 n
    const int a = blockIdx.x, r = blockIdx.y;
    const size_t nn = (size_t)n * n;
    S += a * nn; Si += a * nn; E += (size_t)a * n;
    double2 *xs = buf, *ws = buf + n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = x[((size_t)a * n + i) * nrhs + r];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double2 s = mk<double>(0, 0);
        for (int j = 0; j < n; ++j) s = cfma<double>(Si[(size_t)j * n + i], xs[j], s);
        // s / (1 + i alpha (E_i + shift))
        const double2 e = E[i];
        const double2 d = mk<double>(1.0 - alpha.y * (e.x + shift) - alpha.x * e.y,
                                     alpha.x * (e.x + shift) - alpha.y * e.y);
        const double dd = d.x * d.x + d.y * d.y;
        ws[i] = mk<double>((s.x * d.x + s.y * d.y) / dd, (s.y * d.x - s.x * d.y) / dd);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double2 s = mk<double>(0, 0);
        for (int j = 0; j < n; ++j) s = cfma<double>(S[(size_t)j * n + i], ws[j], s);
        y[((size_t)a * n + i) * nrhs + r] = s;
    }
}

}  // namespace

extern "C" int he_ionic_create(he_ionic **out, int ndof, int nrhs, int nmat, long long nnz, const int *ptr,
                               const int *col, const double *data)
{
    if (!out || !ptr || !col || !data) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    *out = nullptr;
    if (ndof < 1 || nnz < 1 || nmat < 1 || nmat > IONIC_MAX_MATS || nrhs < 1 || nrhs > IONIC_MAX_RHS)
        return he_fail(HE_ERR_ARG, "ionic operator: 1 <= matrices <= 16, 1 <= right-hand sides <= 16", __FILE__, __LINE__);
    if (ptr[0] != 0 || ptr[ndof] != nnz) return he_fail(HE_ERR_SHAPE, "ionic CSR pointer does not span nnz", __FILE__, __LINE__);
    for (long long e = 0; e < nnz; ++e)
        if (col[e] < 0 || col[e] >= ndof) return he_fail(HE_ERR_SHAPE, "ionic CSR column out of range", __FILE__, __LINE__);
    he_ionic *h = new he_ionic();
    h->ndof = ndof; h->nrhs = nrhs; h->nmat = nmat; h->nnz = nnz;
    cudaError_t e = cudaGetDevice(&h->device);
    if (e == cudaSuccess) e = cudaMalloc(&h->ptr, (ndof + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&h->col, nnz * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&h->data, (size_t)nmat * nnz * sizeof(double2));
    if (e == cudaSuccess) e = cudaMemcpy(h->ptr, ptr, (ndof + 1) * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->col, col, nnz * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->data, data, (size_t)nmat * nnz * sizeof(double2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        he_set_error(cudaGetErrorString(e), __FILE__, __LINE__);
        delete h;
        return HE_ERR_CUDA;
    }
    *out = h;
    return HE_OK;
}

extern "C" int he_ionic_set_preconditioner(he_ionic *h, int na, int n, const double *S, const double *Si, const double *E)
{
    if (!h || !S || !Si || !E) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (na < 1 || n < 1 || (long long)na * n != h->ndof)
        return he_fail(HE_ERR_SHAPE, "preconditioner blocks must tile the ionic vector", __FILE__, __LINE__);
    if ((size_t)2 * n * sizeof(double2) > 48 * 1024) return he_fail(HE_ERR_SHAPE, "ionic block too large", __FILE__, __LINE__);
    cudaFree(h->S); cudaFree(h->Si); cudaFree(h->E);
    h->S = h->Si = h->E = nullptr;
    const size_t mat = (size_t)na * n * n * sizeof(double2);
    HE_CUDA_TRY(cudaMalloc(&h->S, mat));
    HE_CUDA_TRY(cudaMalloc(&h->Si, mat));
    HE_CUDA_TRY(cudaMalloc(&h->E, (size_t)na * n * sizeof(double2)));
    HE_CUDA_TRY(cudaMemcpy(h->S, S, mat, cudaMemcpyHostToDevice));
    HE_CUDA_TRY(cudaMemcpy(h->Si, Si, mat, cudaMemcpyHostToDevice));
    HE_CUDA_TRY(cudaMemcpy(h->E, E, (size_t)na * n * sizeof(double2), cudaMemcpyHostToDevice));
    h->na = na; h->n = n;
    return HE_OK;
}

extern "C" int he_ionic_apply(he_ionic *h, const double *coef, int ncoef, const void *x, void *y, double alpha_re,
                              double alpha_im, double shift, int shifted, void *stream)
{
    if (!h || !coef || !x || !y) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (ncoef != h->nmat) return he_fail(HE_ERR_ARG, "one coefficient per matrix plane", __FILE__, __LINE__);
    Coefs cf = {};
    for (int k = 0; k < ncoef; ++k) cf.c[k] = coef[k];
    const int warps = 8;
    ionic_apply_kernel<<<(h->ndof + warps - 1) / warps, 32 * warps, 0, static_cast<cudaStream_t>(stream)>>>(
        h->ndof, h->nrhs, h->nmat, h->nnz, h->ptr, h->col, h->data, cf, static_cast<const double2 *>(x),
        static_cast<double2 *>(y), make_double2(alpha_re, alpha_im), shift, shifted);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

extern "C" int he_ionic_precondition(he_ionic *h, const void *x, void *y, double alpha_re, double alpha_im, double shift,
                                     void *stream)
{
    if (!h || !x || !y) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (!h->S) return he_fail(HE_ERR_ARG, "no preconditioner set", __FILE__, __LINE__);
    const dim3 grid(h->na, h->nrhs);
    ionic_precondition_kernel<<<grid, 256, 2 * h->n * sizeof(double2), static_cast<cudaStream_t>(stream)>>>(
        h->n, h->nrhs, h->S, h->Si, h->E, static_cast<const double2 *>(x), static_cast<double2 *>(y),
        make_double2(alpha_re, alpha_im), shift);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

extern "C" int he_ionic_destroy(he_ionic *h)
{
    delete h;
    return HE_OK;
}
