// Device-driven GMRES for the shifted Pade systems of CF4 (python/implicit.py:45-74, 76-89):
//   (I + i alpha (H(field) - E_ref)) s = b,  right preconditioned by M (the separable resolvent
//   or the Jacobi diagonal), flexible when the preconditioner is complex64.
//
// Every decision the reference takes on the host is taken on the device, so one solve is
// enqueued without host waits and read back once:
//   * least squares by Givens rotations updated one column per iteration (one thread): the
//     rotated right-hand side gives the residual estimate |g_{j+1}| of the reference's
//     lstsq at every check point (every 4 iterations, flexible: 2, and at the restart
//     length), and the rotated columns give y by back substitution when a candidate is tried;
//   * a candidate x + M(Q y) (flexible: x + Z y) is accepted only on its TRUE residual
//     ||b - A x|| / ||b|| <= tol, computed on the device; otherwise the cycle goes on, or
//     restarts from the candidate at a breakdown (h < 1e-14) or at the restart length;
//   * a breakdown at an iteration that is not a check point stops the cycle's iterations
//     and the candidate is tried at the next enqueued check point, with the same dimension.
// Kernels read three gate words: the workspace status `done` (the cycle is over: iterations
// return at once), `skip_try` (no candidate pending) and `skip_accept` (no accepted candidate
// to copy).  A solve is enqueued in segments: first up to the dimension earlier solves of the
// same configuration needed, then (if the status read shows it still running) the rest of
// the cycle and further cycles; the launches, and so the results, do not depend on the split.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "krylov.cuh"
#include "operator.cuh"

namespace he {

struct GmresHeader {          // read back by the host after each segment
    int skip_try;             // 1 unless a candidate test is pending
    int skip_accept;          // 1 unless the last candidate was accepted (to be copied into x)
    int solved;               // the true residual met the tolerance
    int breakdown;            // h < 1e-14 in this cycle
    int m;                    // dimension of the pending / last candidate
    int iterations;           // inner iterations so far (the reference's count)
    int cycles;               // cycles started
    unsigned int ticket;      // last-block counter of the accept copy
    double bnorm, beta, estimate, true_residual;
};

struct GmresState {
    GmresHeader h;
    double2 g[KRYLOV_MAXDIM + 1];             // rotated right-hand side
    double c[KRYLOV_MAXDIM];                  // Givens cosines (real)
    double2 s[KRYLOV_MAXDIM];                 // Givens sines
    double2 y[KRYLOV_MAXDIM];                 // least-squares solution of the pending candidate
    double2 R[KRYLOV_MAXDIM * KRYLOV_MAXDIM]; // rotated Hessenberg columns (upper triangle), ld KRYLOV_MAXDIM
};

namespace {

constexpr int GM_BLOCKS = KRYLOV_BLOCKS;
constexpr int GM_THREADS = KRYLOV_THREADS;

__device__ __forceinline__ bool gated(const int *gate) { return gate && *gate; }

// r = b - t (r may be null) and per-block |b - t|^2 (t null: |b|^2)
__global__ void __launch_bounds__(GM_THREADS)
gm_residual_kernel(size_t n, const double2 *__restrict__ b, const double2 *__restrict__ t, double2 *__restrict__ r,
                   double *__restrict__ partial, const int *gate)
{
    if (gated(gate)) return;
    double s = 0;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const double2 v = t ? csub<double>(b[p], t[p]) : b[p];
        if (r) r[p] = v;
        s += cabs2<double>(v);
    }
    __shared__ double red[GM_THREADS / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tt = 0;
        for (int w = 0; w < GM_THREADS / 32; ++w) tt += red[w];
        partial[blockIdx.x] = tt;
    }
}

// ||b|| of the solve; clears the solve-level state.
__global__ void gm_init_kernel(const double *__restrict__ partial, int nb, GmresState *gs)
{
    const double s = warp_fixed_sum(partial, nb, 1);
    if (threadIdx.x != 0) return;
    GmresHeader h{};
    h.skip_try = 1;
    h.skip_accept = 1;
    h.bnorm = sqrt(s);
    gs->h = h;
}

// Cycle start: beta = ||r0||; converged at once when beta <= tol ||b|| (x is the answer),
// else q0 = r0 / beta follows (gm_scale_kernel) and the rotations start from g = beta e1.
__global__ void gm_start_kernel(const double *__restrict__ partial, int nb, KrylovStatus *st, GmresState *gs, double tol)
{
    const double s = warp_fixed_sum(partial, nb, 1);
    if (threadIdx.x != 0) return;
    const double beta = sqrt(s);
    memset(st, 0, sizeof(KrylovStatus));
    st->beta = beta;
    st->hnext = beta;
    GmresHeader &h = gs->h;
    h.beta = beta;
    h.cycles += 1;
    h.breakdown = 0;
    h.skip_try = 1;
    h.skip_accept = 1;
    for (int k = 0; k <= KRYLOV_MAXDIM; ++k) gs->g[k] = mk<double>(0, 0);
    gs->g[0] = mk<double>(beta, 0);
    if (beta <= tol * h.bnorm) {
        h.solved = 1;
        h.true_residual = h.bnorm > 0 ? beta / h.bnorm : 0.0;
        st->done = 1;
    }
}

// x *= 1 / status.hnext (skipped once the cycle is over)
__global__ void __launch_bounds__(GM_THREADS)
gm_scale_kernel(size_t n, double2 *x, const KrylovStatus *st)
{
    if (st->done) return;
    const double s = 1.0 / st->hnext;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        x[p] = cscale<double>(s, x[p]);
}

// Column j of the Hessenberg (after CGS2 and the norm): apply the previous rotations, form
// the rotation that zeroes h_{j+1,j}, update g and the residual estimate |g_{j+1}|, and
// decide whether a candidate is tried (check point with a small estimate, the restart
// length, or a breakdown).  One thread.
__global__ void gm_givens_kernel(const double2 *__restrict__ H, int ld, int j, int restart, int checkpoint, double tol,
                                 KrylovStatus *st, GmresState *gs)
{
    if (threadIdx.x != 0 || st->done) return;
    GmresHeader &hd = gs->h;
    hd.iterations += 1;
    double2 *col = gs->R + (size_t)j * KRYLOV_MAXDIM;
    for (int i = 0; i <= j; ++i) col[i] = H[(size_t)j * ld + i];
    const double hsub = H[(size_t)j * ld + j + 1].x;      // h_{j+1,j} = ||v|| (real)
    for (int i = 0; i < j; ++i) {                          // [c s; -conj(s) c] on rows i, i+1
        const double2 a = col[i], b = col[i + 1], s = gs->s[i];
        const double c = gs->c[i];
        col[i] = cfma<double>(s, b, cscale<double>(c, a));
        col[i + 1] = csub<double>(cscale<double>(c, b), cmul<double>(mk<double>(s.x, -s.y), a));
    }
    const double2 a = col[j];
    const double amag = sqrt(cabs2<double>(a));
    const double rho = sqrt(amag * amag + hsub * hsub);
    double c;
    double2 s;
    if (amag == 0.0) {
        c = 0.0;
        s = mk<double>(1.0, 0.0);
        col[j] = mk<double>(hsub, 0.0);
    } else {
        const double2 phase = mk<double>(a.x / amag, a.y / amag);
        c = amag / rho;
        s = cscale<double>(hsub / rho, phase);              // phase * conj(h) / rho, h real
        col[j] = cscale<double>(rho, phase);
    }
    gs->c[j] = c;
    gs->s[j] = s;
    const double2 gj = gs->g[j];
    gs->g[j] = cscale<double>(c, gj);
    gs->g[j + 1] = cmul<double>(mk<double>(-s.x, s.y), gj);
    hd.estimate = sqrt(cabs2<double>(gs->g[j + 1]));
    bool trial = false;
    if (hsub < 1e-14) {                                    // breakdown: the cycle's iterations stop here
        hd.breakdown = 1;
        st->done = 1;
        trial = true;
    } else if (checkpoint && (hd.estimate < tol * hd.bnorm || j + 1 == restart)) {
        trial = true;
    }
    if (!trial) return;
    const int m = j + 1;
    hd.m = m;
    for (int i = m - 1; i >= 0; --i) {                     // R y = g by back substitution
        double2 acc = gs->g[i];
        for (int k = i + 1; k < m; ++k)
            acc = csub<double>(acc, cmul<double>(gs->R[(size_t)k * KRYLOV_MAXDIM + i], gs->y[k]));
        const double2 d = gs->R[(size_t)i * KRYLOV_MAXDIM + i];
        const double dd = cabs2<double>(d);
        gs->y[i] = mk<double>((acc.x * d.x + acc.y * d.y) / dd, (acc.y * d.x - acc.x * d.y) / dd);
    }
    hd.skip_try = 0;
}

// out = sum_{k < m} y_k V_k (m and y from the state); skipped unless a candidate is pending
__global__ void __launch_bounds__(GM_THREADS)
gm_combine_kernel(const double2 *__restrict__ V, size_t n, size_t stride, const GmresState *gs,
                  double2 *__restrict__ out)
{
    if (gs->h.skip_try) return;
    const int m = gs->h.m;
    __shared__ double2 ys[KRYLOV_MAXDIM];
    for (int k = threadIdx.x; k < m; k += blockDim.x) ys[k] = gs->y[k];
    __syncthreads();
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        double2 acc = mk<double>(0, 0);
        for (int k = 0; k < m; ++k) acc = cfma<double>(ys[k], V[(size_t)k * stride + p], acc);
        out[p] = acc;
    }
}

// cand = x + d (pending candidate only)
__global__ void __launch_bounds__(GM_THREADS)
gm_candidate_kernel(size_t n, const double2 *__restrict__ x, const double2 *__restrict__ d, double2 *__restrict__ cand,
                    const int *gate)
{
    if (gated(gate)) return;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        cand[p] = cadd<double>(x[p], d[p]);
}

// The candidate's true relative residual decides: solved; or restart from it (breakdown or
// restart length); or carry on with the cycle.
__global__ void gm_decide_kernel(const double *__restrict__ partial, int nb, int restart, double tol, KrylovStatus *st,
                                 GmresState *gs)
{
    if (gs->h.skip_try) return;
    const double s = warp_fixed_sum(partial, nb, 1);
    if (threadIdx.x != 0) return;
    GmresHeader &h = gs->h;
    h.true_residual = sqrt(s) / h.bnorm;
    h.skip_accept = 1;
    if (h.true_residual <= tol) {
        h.solved = 1;
        h.skip_accept = 0;
        st->done = 1;
    } else if (h.breakdown || h.m == restart) {
        h.skip_accept = 0;
        st->done = 1;
    }
    h.skip_try = 1;
}

// x = cand when the candidate was accepted; the last block to finish clears the flag
__global__ void __launch_bounds__(GM_THREADS)
gm_accept_kernel(size_t n, const double2 *__restrict__ cand, double2 *__restrict__ x, GmresState *gs)
{
    if (gs->h.skip_accept) return;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        x[p] = cand[p];
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&gs->h.ticket, 1u) == gridDim.x - 1) {
            gs->h.skip_accept = 1;
            gs->h.ticket = 0;
            __threadfence();
        }
    }
}

// y = x / (1 + i alpha (d + shift))  (the reference's Jacobi preconditioner), gated
__global__ void __launch_bounds__(GM_THREADS)
gm_jacobi_kernel(size_t n, const double2 *__restrict__ d, double2 alpha, double shift, const double2 *__restrict__ x,
                 double2 *__restrict__ y, const int *gate)
{
    if (gated(gate)) return;
    const double2 ia = mk<double>(-alpha.y, alpha.x);
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const double2 den = cfma<double>(ia, mk<double>(d[p].x + shift, d[p].y), mk<double>(1, 0));
        const double q = cabs2<double>(den);
        const double2 v = x[p];
        y[p] = mk<double>((v.x * den.x + v.y * den.y) / q, (v.y * den.x - v.x * den.y) / q);
    }
}

__global__ void __launch_bounds__(GM_THREADS)
gm_to_c64_kernel(size_t n, const double2 *__restrict__ x, float2 *__restrict__ y, const int *gate)
{
    if (gated(gate)) return;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        y[p] = make_float2((float)x[p].x, (float)x[p].y);
}

__global__ void __launch_bounds__(GM_THREADS)
gm_to_c128_kernel(size_t n, const float2 *__restrict__ x, double2 *__restrict__ y, const int *gate)
{
    if (gated(gate)) return;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        y[p] = make_double2((double)x[p].x, (double)x[p].y);
}

}  // namespace
}  // namespace he

using namespace he;

// Per-workspace GMRES buffers (allocated on first use, freed with the workspace).
struct he_gmres_buffers {
    GmresState *state = nullptr;
    GmresHeader *host = nullptr;          // pinned mirror of the header
    KrylovStatus *host_status = nullptr;
    double2 *t = nullptr, *z = nullptr, *c = nullptr, *d = nullptr, *cand = nullptr;
    double2 *step = nullptr;              // he_cf4_step: the solution of the current Pade solve
    float2 *s32[2] = {nullptr, nullptr};
    size_t n = 0;
    long long hint_key = 0;
    int iters_seen = 0;                   // most iterations a cycle of that configuration needed
    ~he_gmres_buffers()
    {
        cudaFree(state); cudaFree(t); cudaFree(z); cudaFree(c); cudaFree(d); cudaFree(cand); cudaFree(step);
        cudaFree(s32[0]); cudaFree(s32[1]);
        if (host) cudaFreeHost(host);
        if (host_status) cudaFreeHost(host_status);
    }
};

void he_gmres_buffers_free(he_gmres_buffers *b) { delete b; }

namespace {

struct Solve {
    he_krylov *k;
    he_gmres_buffers *gb;
    he_handle op;
    he_separable *sep;
    const double2 *diag;
    const double2 *b;
    double2 *x;
    double field[3];
    double2 alpha;
    double eref, shift, tol;
    int restart, precision;
    cudaStream_t s;
};

const dim3 kGrid(GM_BLOCKS), kThreads(GM_THREADS);

// out = A in = in + i alpha (H in - E_ref in), gated (complex64 operator: through the
// complex64 buffers)
int apply_A(const Solve &v, const double2 *in, double2 *out, const int *gate)
{
    const size_t n = v.k->n;
    if (v.precision == HE_C64) {
        gm_to_c64_kernel<<<kGrid, kThreads, 0, v.s>>>(n, in, v.gb->s32[0], gate);
        int rc = apply_shifted_gated(v.op, v.gb->s32[0], v.gb->s32[1], v.field, 1, v.alpha.x, v.alpha.y, v.eref, HE_C64,
                                     gate, v.s);
        if (rc) return rc;
        gm_to_c128_kernel<<<kGrid, kThreads, 0, v.s>>>(n, v.gb->s32[1], out, gate);
        return HE_OK;
    }
    return apply_shifted_gated(v.op, in, out, v.field, 1, v.alpha.x, v.alpha.y, v.eref, HE_C128, gate, v.s);
}

int apply_M(const Solve &v, const double2 *in, double2 *out, const int *gate)
{
    if (v.sep) return separable_apply_gated(v.sep, in, out, v.alpha, v.shift, gate, v.s);
    gm_jacobi_kernel<<<kGrid, kThreads, 0, v.s>>>(v.k->n, v.diag, v.alpha, v.shift, in, out, gate);
    return HE_OK;
}

int enqueue_cycle_start(const Solve &v)
{
    he_krylov *k = v.k;
    double2 *q0 = k->Q;
    int rc = apply_A(v, v.x, v.gb->t, nullptr);
    if (rc) return rc;
    gm_residual_kernel<<<kGrid, kThreads, 0, v.s>>>(k->n, v.b, v.gb->t, q0, k->norm_partial, nullptr);
    gm_start_kernel<<<1, 32, 0, v.s>>>(k->norm_partial, GM_BLOCKS, k->status, v.gb->state, v.tol);
    gm_scale_kernel<<<kGrid, kThreads, 0, v.s>>>(k->n, q0, k->status);
    HE_CUDA_TRY(cudaMemsetAsync(k->H, 0, sizeof(double2) * k->hs(), v.s));
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

int enqueue_iterations(const Solve &v, int j0, int j1)
{
    he_krylov *k = v.k;
    const int ld = k->maxdim + 1, cadence = k->flexible ? 2 : 4;
    const int *done = &k->status->done;
    GmresState *gs = v.gb->state;
    const int *skip_try = &gs->h.skip_try;
    int rc = HE_OK;
    for (int j = j0; j < j1 && !rc; ++j) {
        double2 *qj = k->Q + (size_t)j * k->n, *q1 = k->Q + (size_t)(j + 1) * k->n;
        double2 *zj = k->flexible ? k->Z + (size_t)j * k->n : v.gb->z;
        if ((rc = apply_M(v, qj, zj, done))) break;
        if ((rc = apply_A(v, zj, q1, done))) break;
        // CGS2: up to 16 basis vectors as the fused sweeps (projection; update + second
        // projection + h; the second update and 1/h after the rotation step), beyond as
        // separate projection / update launches
        const bool fused = j + 1 <= KRYLOV_FUSED;
        if (fused) rc = krylov_cgs2_fused(k, j + 1, q1, j, v.s, 1e-14);
        else rc = krylov_cgs2(k, j + 1, q1, k->H + (size_t)j * ld, k->H + (size_t)j * ld + j + 1, v.s, 1e-14);
        if (rc) break;
        const bool checkpoint = (j + 1) % cadence == 0 || j + 1 == v.restart;
        gm_givens_kernel<<<1, 32, 0, v.s>>>(k->H, ld, j, v.restart, checkpoint, v.tol, k->status, gs);
        if (checkpoint) {     // the candidate test (runs only when the rotation step asked for it)
            gm_combine_kernel<<<kGrid, kThreads, 0, v.s>>>(k->flexible ? k->Z : k->Q, k->n, k->n, gs, v.gb->c);
            const double2 *dir = v.gb->c;
            if (!k->flexible) {
                if ((rc = apply_M(v, v.gb->c, v.gb->d, skip_try))) break;
                dir = v.gb->d;
            }
            gm_candidate_kernel<<<kGrid, kThreads, 0, v.s>>>(k->n, v.x, dir, v.gb->cand, skip_try);
            if ((rc = apply_A(v, v.gb->cand, v.gb->t, skip_try))) break;
            gm_residual_kernel<<<kGrid, kThreads, 0, v.s>>>(k->n, v.b, v.gb->t, nullptr, k->norm_partial, skip_try);
            gm_decide_kernel<<<1, 32, 0, v.s>>>(k->norm_partial, GM_BLOCKS, v.restart, v.tol, k->status, gs);
            gm_accept_kernel<<<kGrid, kThreads, 0, v.s>>>(k->n, v.gb->cand, v.x, gs);
        }
        if (j + 1 < v.restart) {
            if (fused) {
                if ((rc = krylov_next(k, j + 1, q1, v.s))) break;
            } else {
                gm_scale_kernel<<<kGrid, kThreads, 0, v.s>>>(k->n, q1, k->status);
            }
        }
        HE_CUDA_TRY(cudaGetLastError());
    }
    return rc;
}

int read_state(const Solve &v)
{
    HE_CUDA_TRY(cudaMemcpyAsync(v.gb->host, &v.gb->state->h, sizeof(GmresHeader), cudaMemcpyDeviceToHost, v.s));
    HE_CUDA_TRY(cudaMemcpyAsync(v.gb->host_status, v.k->status, sizeof(KrylovStatus), cudaMemcpyDeviceToHost, v.s));
    HE_CUDA_TRY(cudaStreamSynchronize(v.s));
    return HE_OK;
}

int buffers(he_krylov *k, int precision, he_gmres_buffers **out)
{
    he_gmres_buffers *gb = k->gmres;
    if (!gb) {
        gb = new he_gmres_buffers();
        gb->n = k->n;
        cudaError_t e = cudaMalloc(&gb->state, sizeof(GmresState));
        for (double2 **p : {&gb->t, &gb->z, &gb->c, &gb->d, &gb->cand})
            if (e == cudaSuccess) e = cudaMalloc(p, k->n * sizeof(double2));
        if (e == cudaSuccess) e = cudaMallocHost(&gb->host, sizeof(GmresHeader));
        if (e == cudaSuccess) e = cudaMallocHost(&gb->host_status, sizeof(KrylovStatus));
        if (e != cudaSuccess) {
            delete gb;
            he_set_error(cudaGetErrorString(e), __FILE__, __LINE__);
            return HE_ERR_CUDA;
        }
        k->gmres = gb;
    }
    if (precision == HE_C64 && !gb->s32[0])
        for (int q = 0; q < 2; ++q) HE_CUDA_TRY(cudaMalloc(&gb->s32[q], k->n * sizeof(float2)));
    *out = gb;
    return HE_OK;
}

}  // namespace

extern "C" int he_gmres_shifted(he_krylov *k, he_handle op, he_separable *sep, const void *diag, const void *b, void *x,
                                const double *field, double alpha_re, double alpha_im, double e_ref, double shift,
                                double tol, int restart, int max_restarts, int precision, int *iterations,
                                double *residual, void *stream)
{
    if (!k || !op || !b || !x || !field || (!sep && !diag) || b == x)
        return he_fail(HE_ERR_ARG, "bad GMRES argument", __FILE__, __LINE__);
    if (k->count != 1) return he_fail(HE_ERR_ARG, "GMRES needs a single-instance workspace", __FILE__, __LINE__);
    if (restart < 1 || restart > k->maxdim || max_restarts < 1)
        return he_fail(HE_ERR_ARG, "restart length exceeds the workspace", __FILE__, __LINE__);
    if (precision != HE_C128 && precision != HE_C64) return he_fail(HE_ERR_ARG, "bad precision", __FILE__, __LINE__);
    if ((size_t)op->n * op->n * op->nc != k->n) return he_fail(HE_ERR_SHAPE, "workspace size != operator size", __FILE__, __LINE__);
    he_gmres_buffers *gb = nullptr;
    int rc = buffers(k, precision, &gb);
    if (rc) return rc;
    Solve v{k, gb, op, sep, static_cast<const double2 *>(diag), static_cast<const double2 *>(b),
            static_cast<double2 *>(x), {field[0], field[1], field[2]}, mk<double>(alpha_re, alpha_im), e_ref, shift,
            tol, restart, precision, static_cast<cudaStream_t>(stream)};
    // x0 = b (python/implicit.py:47) and ||b||
    HE_CUDA_TRY(cudaMemcpyAsync(v.x, v.b, k->n * sizeof(double2), cudaMemcpyDeviceToDevice, v.s));
    gm_residual_kernel<<<kGrid, kThreads, 0, v.s>>>(k->n, v.b, nullptr, nullptr, k->norm_partial, nullptr);
    gm_init_kernel<<<1, 32, 0, v.s>>>(k->norm_partial, GM_BLOCKS, gb->state);
    // speculative segment length: the iterations earlier solves of this configuration needed
    const long long key = (long long)(reinterpret_cast<uintptr_t>(op) ^ (reinterpret_cast<uintptr_t>(sep) << 1) ^
                                      ((uintptr_t)precision << 2) ^ ((uintptr_t)restart << 8) ^
                                      ((uintptr_t)k->flexible << 20));
    if (gb->hint_key != key) { gb->hint_key = key; gb->iters_seen = 0; }
    const int cadence = k->flexible ? 2 : 4;
    for (int cycle = 0; cycle < max_restarts; ++cycle) {
        if ((rc = enqueue_cycle_start(v))) return rc;
        int j = 0;
        int first = restart;
        if (gb->iters_seen > 0) first = std::min(restart, (gb->iters_seen + cadence - 1) / cadence * cadence);
        while (j < restart) {
            // a solve that outruns the hint continues in doubling segments
            const int end = j == 0 ? first : std::min(restart, j + std::max(cadence, j));
            if ((rc = enqueue_iterations(v, j, end))) return rc;
            if ((rc = read_state(v))) return rc;
            j = end;
            if (gb->host->solved || gb->host_status->done) break;
        }
        if (gb->host->solved) {
            // the hint follows first cycles that converged; a solve that restarts runs its
            // first cycle to the restart length in two segments anyway, and must not make
            // every later solve enqueue whole cycles
            const int in_cycle = gb->host->m;
            if (cycle == 0 && in_cycle > gb->iters_seen) gb->iters_seen = in_cycle;
            if (iterations) *iterations = gb->host->iterations;
            if (residual) *residual = gb->host->true_residual;
            return HE_OK;
        }
    }
    if (iterations) *iterations = gb->host->iterations;
    if (residual) *residual = gb->host->true_residual;
    char msg[128];
    snprintf(msg, sizeof(msg), "GMRES did not converge: residual=%.3e, iterations=%d", gb->host->true_residual,
             gb->host->iterations);
    return he_fail(HE_ERR_NOCONV, msg, __FILE__, __LINE__);
}

// Iterations the first segment of the next solve on this workspace enqueues (0: a whole
// cycle), and the configuration key the hint belongs to.
extern "C" int he_gmres_segment_hint(he_krylov *k, int *iterations, long long *key)
{
    if (!k || !iterations) return he_fail(HE_ERR_ARG, "null GMRES hint argument", __FILE__, __LINE__);
    const he_gmres_buffers *gb = k->gmres;
    *iterations = gb ? gb->iters_seen : 0;
    if (key) *key = gb ? gb->hint_key : 0;
    return HE_OK;
}

// Host arithmetic of a CF4 step (python/implicit.py:91-109, :76-89) from the vector
// potentials at the two Gauss points (fields: 2 x 3).  out[5 e .. 5 e + 4] for exponential
// e = 0, 1 (field weights (A2, A1), (A1, A2)): the effective field (3), the preconditioner
// shift a2 |A_eff|^2 - e_ref, and the phase angle -dt (a2 (w . |A|^2 - |A_eff|^2 / 2) +
// e_ref / 2); out[10 + 2 r], out[11 + 2 r]: alpha = (dt / 2) / (3 + i sigma_r sqrt 3), sigma
// = +1, -1.
extern "C" int he_cf4_coefficients(const double *fields, double dt, double e_ref, double a2, double *out)
{
    if (!fields || !out) return he_fail(HE_ERR_ARG, "null CF4 coefficient argument", __FILE__, __LINE__);
    const double sqrt3 = std::sqrt(3.0);
    const double A1 = (3 - 2 * sqrt3) / 12, A2 = (3 + 2 * sqrt3) / 12;
    const double weights[2][2] = {{A2, A1}, {A1, A2}};
    double sumsq[2];
    for (int a = 0; a < 2; ++a) sumsq[a] = fields[3 * a] * fields[3 * a] + fields[3 * a + 1] * fields[3 * a + 1] +
                                           fields[3 * a + 2] * fields[3 * a + 2];
    for (int e = 0; e < 2; ++e) {
        const double *w = weights[e];
        double *o = out + 5 * e, effsq = 0;
        for (int j = 0; j < 3; ++j) {
            o[j] = 2 * (w[0] * fields[j] + w[1] * fields[3 + j]);
            effsq += o[j] * o[j];
        }
        const double correction = a2 * (w[0] * sumsq[0] + w[1] * sumsq[1] - .5 * effsq);
        o[3] = a2 * effsq - e_ref;
        o[4] = -dt * (correction + e_ref / 2);
    }
    for (int r = 0; r < 2; ++r) {
        // (dt / 2) / (3 + i sigma sqrt 3) = (dt / 2) (3 - i sigma sqrt 3) / 12
        const double sigma = r == 0 ? 1 : -1;
        out[10 + 2 * r] = dt / 2 * 3 / 12;
        out[11 + 2 * r] = -sigma * dt / 2 * sqrt3 / 12;
    }
    return HE_OK;
}

extern "C" int he_vec_axpby(long long n, double a_re, double a_im, const void *x, double b_re, double b_im,
                            const void *y, void *out, void *stream);

// One commutator-free fourth-order Magnus step (python/implicit.py:91-109): two
// exponentials with the field weights (A2, A1) and (A1, A2) of the Gauss-point vector
// potentials, each a [2/2] Pade pair of shifted solves (I + i alpha (H(A_eff) - e_ref)) s = x,
// alpha = (dt / 2) / (3 +- i sqrt 3), x <- 2 s - x (python/implicit.py:76-89), each solve the
// device GMRES above, followed by the phase exp(-i dt (a2 (w . |A|^2 - |A_eff|^2 / 2) + e_ref / 2))
// (the coefficients of he_cf4_coefficients).
extern "C" int he_cf4_step(he_krylov *k, he_handle op, he_separable *sep, const void *diag, const void *x, void *y,
                           const double *fields, double dt, double e_ref, double a2, double tol, int restart,
                           int max_restarts, int *iterations, double *residual, void *stream)
{
    if (!k || !op || !x || !y || !fields || x == y || (!sep && !diag))
        return he_fail(HE_ERR_ARG, "bad CF4 step argument", __FILE__, __LINE__);
    if ((size_t)op->n * op->n * op->nc != k->n) return he_fail(HE_ERR_SHAPE, "workspace size != operator size", __FILE__, __LINE__);
    he_gmres_buffers *gb = nullptr;
    int rc = buffers(k, HE_C128, &gb);
    if (rc) return rc;
    if (!gb->step) HE_CUDA_TRY(cudaMalloc(&gb->step, k->n * sizeof(double2)));
    double co[14];
    if ((rc = he_cf4_coefficients(fields, dt, e_ref, a2, co))) return rc;
    const long long n = (long long)k->n;
    int total = 0;
    double worst = 0;
    const void *src = x;
    for (int e = 0; e < 2; ++e) {
        const double *eff = co + 5 * e, shift = co[5 * e + 3], theta = co[5 * e + 4];
        for (int r = 0; r < 2; ++r) {
            int it = 0;
            double res = 0;
            rc = he_gmres_shifted(k, op, sep, diag, src, gb->step, eff, co[10 + 2 * r], co[11 + 2 * r], e_ref, shift, tol,
                                  restart, max_restarts, HE_C128, &it, &res, stream);
            total += it;
            if (res > worst) worst = res;
            if (rc) {
                if (iterations) *iterations = total;
                if (residual) *residual = worst;
                return rc;
            }
            if ((rc = he_vec_axpby(n, 2, 0, gb->step, -1, 0, src, y, stream))) return rc;
            src = y;
        }
        if ((rc = he_vec_axpby(n, std::cos(theta), std::sin(theta), y, 0, 0, y, y, stream))) return rc;
    }
    if (iterations) *iterations = total;
    if (residual) *residual = worst;
    return HE_OK;
}
