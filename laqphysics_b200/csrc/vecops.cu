// Complex128 vector primitives of the GMRES / CF4 drivers (python/implicit.py:45-109):
// axpby, norms with deterministic two-stage reductions, residual norms, Jacobi
// scaling, Hessenberg column transfer and basis combinations with host coefficients.
#include <vector>

#include "common.cuh"
#include "krylov.cuh"
#include "operator.cuh"

namespace he {

__global__ void __launch_bounds__(KRYLOV_THREADS)
axpby_kernel(size_t n, double2 a, const double2 *x, double2 b, const double2 *y, double2 *out)
{
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        out[p] = cfma<double>(a, x[p], cmul<double>(b, y[p]));
}

// r = b - t (written when r != nullptr) and per-block |b - t|^2 (t == nullptr: |b|^2)
__global__ void __launch_bounds__(KRYLOV_THREADS)
residual_kernel(size_t n, const double2 *b, const double2 *t, double2 *r, double *partial)
{
    double s = 0;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const double2 v = t ? csub<double>(b[p], t[p]) : b[p];
        if (r) r[p] = v;
        s += cabs2<double>(v);
    }
    __shared__ double red[KRYLOV_THREADS / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tt = 0;
        for (int w = 0; w < KRYLOV_THREADS / 32; ++w) tt += red[w];
        partial[blockIdx.x] = tt;
    }
}

__global__ void sum_kernel(const double *partial, int nb, double *out)
{
    const double s = warp_fixed_sum(partial, nb, 1);
    if (threadIdx.x == 0) *out = s;
}

// y = x / (1 + i alpha d)   (Jacobi preconditioner of python/implicit.py:80,85)
__global__ void __launch_bounds__(KRYLOV_THREADS)
jacobi_kernel(size_t n, const double2 *d, double2 alpha, double shift, const double2 *x, double2 *y)
{
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const double2 dd = mk<double>(d[p].x + shift, d[p].y);
        const double2 ia = mk<double>(-alpha.y, alpha.x);            // i alpha
        const double2 den = cfma<double>(ia, dd, mk<double>(1, 0));  // 1 + i alpha d
        const double q = cabs2<double>(den);
        const double2 v = x[p];
        y[p] = mk<double>((v.x * den.x + v.y * den.y) / q, (v.y * den.x - v.x * den.y) / q);
    }
}

__global__ void __launch_bounds__(KRYLOV_THREADS)
scale_kernel(size_t n, double s, double2 *x)
{
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        x[p] = cscale<double>(s, x[p]);
}

__global__ void __launch_bounds__(KRYLOV_THREADS)
combine_host_kernel(const double2 *__restrict__ V, size_t n, int m, const double2 *__restrict__ c, double2 *y,
                    int accumulate)
{
    __shared__ double2 cs[KRYLOV_MAXDIM];
    for (int k = threadIdx.x; k < m; k += blockDim.x) cs[k] = c[k];
    __syncthreads();
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        double2 acc = accumulate ? y[p] : mk<double>(0, 0);
        for (int k = 0; k < m; ++k) acc = cfma<double>(cs[k], V[(size_t)k * n + p], acc);
        y[p] = acc;
    }
}

}  // namespace he

using namespace he;

namespace {
thread_local double *g_partial = nullptr;   // per-thread reduction scratch (KRYLOV_BLOCKS + 1 doubles)
thread_local double *g_host = nullptr;
thread_local int g_partial_device = -1;

int reduction_scratch()
{
    int dev = 0;
    HE_CUDA_TRY(cudaGetDevice(&dev));
    if (g_partial && g_partial_device == dev) return HE_OK;
    if (g_partial) cudaFree(g_partial);   // scratch of another device: replace it
    g_partial = nullptr;
    HE_CUDA_TRY(cudaMalloc(&g_partial, (KRYLOV_BLOCKS + 1) * sizeof(double)));
    if (!g_host) HE_CUDA_TRY(cudaMallocHost(&g_host, sizeof(double)));
    g_partial_device = dev;
    return HE_OK;
}
}  // namespace

extern "C" int he_vec_axpby(long long n, double a_re, double a_im, const void *x, double b_re, double b_im,
                            const void *y, void *out, void *stream)
{
    if (n < 0 || !x || !y || !out) return he_fail(HE_ERR_ARG, "bad axpby argument", __FILE__, __LINE__);
    axpby_kernel<<<KRYLOV_BLOCKS, KRYLOV_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(
        (size_t)n, mk<double>(a_re, a_im), static_cast<const double2 *>(x), mk<double>(b_re, b_im),
        static_cast<const double2 *>(y), static_cast<double2 *>(out));
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

// ||b - t|| (t may be NULL: ||b||); r = b - t stored when r != NULL.  Blocks the host.
extern "C" int he_vec_residual_norm(long long n, const void *b, const void *t, void *r, double *norm, void *stream)
{
    if (n < 0 || !b || !norm) return he_fail(HE_ERR_ARG, "bad residual argument", __FILE__, __LINE__);
    int rc = reduction_scratch();
    if (rc) return rc;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    residual_kernel<<<KRYLOV_BLOCKS, KRYLOV_THREADS, 0, s>>>((size_t)n, static_cast<const double2 *>(b),
                                                             static_cast<const double2 *>(t),
                                                             static_cast<double2 *>(r), g_partial);
    sum_kernel<<<1, 32, 0, s>>>(g_partial, KRYLOV_BLOCKS, g_partial + KRYLOV_BLOCKS);
    HE_CUDA_TRY(cudaMemcpyAsync(g_host, g_partial + KRYLOV_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, s));
    HE_CUDA_TRY(cudaStreamSynchronize(s));
    *norm = sqrt(*g_host);
    return HE_OK;
}

extern "C" int he_vec_jacobi(long long n, const void *diag, double alpha_re, double alpha_im, double shift,
                             const void *x, void *y, void *stream)
{
    if (n < 0 || !diag || !x || !y) return he_fail(HE_ERR_ARG, "bad Jacobi argument", __FILE__, __LINE__);
    jacobi_kernel<<<KRYLOV_BLOCKS, KRYLOV_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(
        (size_t)n, static_cast<const double2 *>(diag), mk<double>(alpha_re, alpha_im), shift,
        static_cast<const double2 *>(x), static_cast<double2 *>(y));
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

extern "C" int he_krylov_vector(he_krylov *k, int which, int j, void **ptr);

extern "C" int he_krylov_scale(he_krylov *k, int which, int j, double s, void *stream)
{
    void *p = nullptr;
    int rc = he_krylov_vector(k, which, j, &p);
    if (rc) return rc;
    scale_kernel<<<KRYLOV_BLOCKS, KRYLOV_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(k->n, s,
                                                                                          static_cast<double2 *>(p));
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

// Copy H[0..rows) of column j (rows <= maxdim+1) to host memory (interleaved complex).  Blocks.
extern "C" int he_krylov_hessenberg(he_krylov *k, int j, int rows, void *out, void *stream)
{
    if (!k || !out || j < 0 || j >= k->maxdim || rows < 1 || rows > k->maxdim + 1)
        return he_fail(HE_ERR_ARG, "bad Hessenberg request", __FILE__, __LINE__);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    HE_CUDA_TRY(cudaMemcpyAsync(out, k->H + (size_t)j * (k->maxdim + 1), rows * sizeof(double2),
                                cudaMemcpyDeviceToHost, s));
    HE_CUDA_TRY(cudaStreamSynchronize(s));
    return HE_OK;
}

// Zero the Hessenberg matrix (start of a GMRES cycle).
extern "C" int he_krylov_reset(he_krylov *k, void *stream)
{
    if (!k) return he_fail(HE_ERR_ARG, "null workspace", __FILE__, __LINE__);
    HE_CUDA_TRY(cudaMemsetAsync(k->H, 0, sizeof(double2) * (k->maxdim + 1) * k->maxdim, static_cast<cudaStream_t>(stream)));
    HE_CUDA_TRY(cudaMemsetAsync(k->status, 0, sizeof(KrylovStatus), static_cast<cudaStream_t>(stream)));
    return HE_OK;
}

// y (+)= sum_{k<m} V_k c_k with V = Q (which = 0) or Z (which = 1) and host coefficients c.
extern "C" int he_krylov_combine_coef(he_krylov *k, int which, int m, const void *coef, void *y, int accumulate,
                                      void *stream)
{
    if (!k || !coef || !y || m < 0 || m > k->maxdim || (which == 1 && !k->Z))
        return he_fail(HE_ERR_ARG, "bad combination", __FILE__, __LINE__);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    HE_CUDA_TRY(cudaMemcpyAsync(k->coef, coef, m * sizeof(double2), cudaMemcpyHostToDevice, s));
    combine_host_kernel<<<KRYLOV_BLOCKS, KRYLOV_THREADS, 0, s>>>(which ? k->Z : k->Q, k->n, m, k->coef,
                                                                 static_cast<double2 *>(y), accumulate);
    HE_CUDA_TRY(cudaGetLastError());
    // the host coefficient buffer may be reused by the caller as soon as this returns
    HE_CUDA_TRY(cudaStreamSynchronize(s));
    return HE_OK;
}

// binaryVersion (major * 10 + minor) of a kernel of this library as the runtime loaded it
// on the current device: 100 for code built for sm_100a.
extern "C" int he_binary_version(int *version)
{
    if (!version) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    cudaFuncAttributes attributes;
    HE_CUDA_TRY(cudaFuncGetAttributes(&attributes, (const void *)sum_kernel));
    *version = attributes.binaryVersion;
    return HE_OK;
}

// ---------------------------------------------------------------------------------
// Run diagnostics of python/run3d.py:212-224 on the device (no state copy to the host):
//   real-region norm  sum |u(i,j,c)|^2 f_i f_j   (f = interior weight / |weight|),
//   <g|psi> = sum conj(g) psi,
//   exchange error^2  sum |u(i,j,c) - sign_c u(j,i,x_c)|^2   (x_c the exchanged channel).
// ---------------------------------------------------------------------------------
namespace he {
__global__ void __launch_bounds__(KRYLOV_THREADS)
diagnostics_kernel(int n, int nc, const double2 *__restrict__ psi, const double2 *__restrict__ g,
                   const double *__restrict__ f, const int *__restrict__ xc, const double *__restrict__ sign,
                   double *__restrict__ partial)
{
    const size_t nn = (size_t)n * n, total = nn * nc;
    double norm = 0, ex = 0;
    double2 ov = mk<double>(0, 0);
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(p / nn);
        const size_t q = p - (size_t)c * nn;
        const int i = (int)(q % n), j = (int)(q / n);
        const double2 u = psi[p];
        norm += cabs2<double>(u) * f[i] * f[j];
        if (g) ov = cfma_conj<double>(g[p], u, ov);
        const double2 w = psi[(size_t)xc[c] * nn + (size_t)i * n + j];
        const double s = sign[c];
        ex += cabs2<double>(mk<double>(u.x - s * w.x, u.y - s * w.y));
    }
    double v[4] = {norm, ov.x, ov.y, ex};
    __shared__ double red[4][KRYLOV_THREADS / 32];
    for (int k = 0; k < 4; ++k) {
        double s = v[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = s;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0;
        for (int w = 0; w < KRYLOV_THREADS / 32; ++w) t += red[threadIdx.x][w];
        partial[(size_t)threadIdx.x * KRYLOV_BLOCKS + blockIdx.x] = t;
    }
}

__global__ void diagnostics_sum_kernel(const double *partial, double *out)
{
    const int k = threadIdx.x >> 5;     // one warp per quantity, fixed order
    const double s = warp_fixed_sum(partial + (size_t)k * KRYLOV_BLOCKS, KRYLOV_BLOCKS, 1);
    if ((threadIdx.x & 31) == 0) out[k] = s;
}
}  // namespace he

// out[0] = real-region norm, out[1] + i out[2] = <g|psi> (0 when g is NULL), out[3] = exchange
// error ||u - P12 u|| (host memory, 4 doubles).  f: n doubles, xc: nc ints, sign: nc doubles,
// all device memory; psi, g: complex128 device states.  Blocks the host until done.
extern "C" int he_diagnostics(he_handle h, const void *psi, const void *g, const double *f, const int *xc,
                              const double *sign, double *out, void *stream)
{
    if (!h || !psi || !f || !xc || !sign || !out) return he_fail(HE_ERR_ARG, "bad diagnostics argument", __FILE__, __LINE__);
    static thread_local double *scratch = nullptr, *host = nullptr;
    static thread_local int scratch_device = -1;
    int dev = 0;
    HE_CUDA_TRY(cudaGetDevice(&dev));
    if (!scratch || scratch_device != dev) {
        if (scratch) cudaFree(scratch);
        scratch = nullptr;
        HE_CUDA_TRY(cudaMalloc(&scratch, (4 * KRYLOV_BLOCKS + 4) * sizeof(double)));
        if (!host) HE_CUDA_TRY(cudaMallocHost(&host, 4 * sizeof(double)));
        scratch_device = dev;
    }
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    diagnostics_kernel<<<KRYLOV_BLOCKS, KRYLOV_THREADS, 0, s>>>(h->n, h->nc, static_cast<const double2 *>(psi),
                                                                static_cast<const double2 *>(g), f, xc, sign, scratch);
    diagnostics_sum_kernel<<<1, 128, 0, s>>>(scratch, scratch + 4 * KRYLOV_BLOCKS);
    HE_CUDA_TRY(cudaGetLastError());
    HE_CUDA_TRY(cudaMemcpyAsync(host, scratch + 4 * KRYLOV_BLOCKS, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    HE_CUDA_TRY(cudaStreamSynchronize(s));
    out[0] = host[0];
    out[1] = host[1];
    out[2] = host[2];
    out[3] = sqrt(host[3]);
    return HE_OK;
}
