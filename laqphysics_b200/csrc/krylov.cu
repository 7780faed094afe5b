// Krylov building blocks on the device: classical Gram-Schmidt applied twice (CGS2)
// with deterministic block reductions, the small Hessenberg exponential
// expm(-i dt H_m) in complex128 on one CTA, and the Arnoldi exponential action of
// the reference's python/propagate.py:6-39 / python/torch_backend.py:140-158.
//
// Reductions: every pass writes one partial per (block, basis vector) into the
// workspace's `partial` array; a single-CTA kernel then sums them, one warp per value
// in a fixed order, so results are bitwise reproducible run to run.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "hamiltonian.cuh"
#include "krylov.cuh"
#include "operator.cuh"

namespace he {

__device__ __forceinline__ double2 warp_sum(double2 v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, off);
        v.y += __shfl_down_sync(0xffffffffu, v.y, off);
    }
    return v;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

// Block-wide sum of KT complex accumulators; thread 0 of the block gets the result.
template <int KT>
__device__ __forceinline__ void block_sum(double2 (&acc)[KT], double2 *out)
{
    __shared__ double2 red[KRYLOV_THREADS / 32][KT];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < KT; ++k) {
        const double2 s = warp_sum(acc[k]);
        if (lane == 0) red[warp][k] = s;
    }
    __syncthreads();
    if (threadIdx.x < KT) {
        double2 s = mk<double>(0, 0);
        for (int w = 0; w < KRYLOV_THREADS / 32; ++w) s = cadd<double>(s, red[w][threadIdx.x]);
        out[threadIdx.x] = s;
    }
}

// Batched workspaces: instance b (blockIdx.y of the vector kernels, blockIdx.x of the
// one-CTA-per-instance kernels) owns vector k of the basis at Q + k*qs + b*n (qs = count*n,
// so basis vector k of every instance is one contiguous block), and its own slices of
// H, partial sums, projections, coefficients, scratch and status.

// partial[b*ld + k0 + k] = sum over this block's elements of conj(Q_{k0+k}) v
template <int KT>
__global__ void __launch_bounds__(KRYLOV_THREADS)
multidot_kernel(const double2 *__restrict__ Q, size_t n, size_t qs, int k0, int kc, const double2 *__restrict__ v,
                double2 *__restrict__ partial, int ld, const KrylovStatus *st)
{
    const int inst = blockIdx.y;
    Q += inst * n; v += inst * n; partial += (size_t)inst * gridDim.x * ld;
    if (st) st += inst;
    if (st && st->done) return;
    double2 acc[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) acc[k] = mk<double>(0, 0);
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        const double2 x = v[p];
#pragma unroll
        for (int k = 0; k < KT; ++k)
            if (k < kc) acc[k] = cfma_conj<double>(Q[(size_t)(k0 + k) * qs + p], x, acc[k]);
    }
    __shared__ double2 res[KT];
    block_sum<KT>(acc, res);
    __syncthreads();
    if (threadIdx.x < kc) partial[(size_t)blockIdx.x * ld + k0 + threadIdx.x] = res[threadIdx.x];
}

// z[k] = sum_b partial[b*ld + k] for k < kc (fixed order, one warp per k); optionally
// H[k] += z[k].
__global__ void reduce_partials_kernel(const double2 *__restrict__ partial, int nb, int ld, int kc,
                                       double2 *__restrict__ z, double2 *__restrict__ hcol, size_t hs,
                                       const KrylovStatus *st)
{
    const int inst = blockIdx.x;
    partial += (size_t)inst * nb * ld; z += (size_t)inst * ld;
    if (hcol) hcol += inst * hs;
    if (st) st += inst;
    if (st && st->done) return;
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int k = warp; k < kc; k += nwarps) {
        const double2 s = warp_fixed_sum(partial + k, nb, (size_t)ld);
        if ((threadIdx.x & 31) == 0) {
            z[k] = s;
            if (hcol) hcol[k] = cadd<double>(hcol[k], s);
        }
    }
}

// v -= sum_k Q_k z_k ; optionally per-block |v|^2 partial sums.
__global__ void __launch_bounds__(KRYLOV_THREADS)
update_kernel(const double2 *__restrict__ Q, size_t n, size_t qs, int kc, const double2 *__restrict__ z, int ld,
              double2 *__restrict__ v, double *__restrict__ norm_partial, const KrylovStatus *st)
{
    const int inst = blockIdx.y;
    Q += inst * n; v += inst * n; z += (size_t)inst * ld;
    if (norm_partial) norm_partial += (size_t)inst * gridDim.x;
    if (st) st += inst;
    if (st && st->done) return;
    __shared__ double2 zs[KRYLOV_MAXDIM + 1];
    for (int k = threadIdx.x; k < kc; k += blockDim.x) zs[k] = z[k];
    __syncthreads();
    double nrm = 0;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        double2 x = v[p];
        for (int k = 0; k < kc; ++k) {
            const double2 q = Q[(size_t)k * qs + p];
            x = cfma<double>(mk<double>(-zs[k].x, -zs[k].y), q, x);
        }
        v[p] = x;
        nrm += cabs2<double>(x);
    }
    if (norm_partial) {
        __shared__ double red[KRYLOV_THREADS / 32];
        const double s = warp_sum(nrm);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int w = 0; w < KRYLOV_THREADS / 32; ++w) t += red[w];
            norm_partial[blockIdx.x] = t;
        }
    }
}

// Second CGS pass fused with the first update: v' = v - sum_k Q_k z_k is written and, in
// the same sweep, partial[b*ld + k] = sum over the block of conj(Q_k) v' (k < kc <= KT).
// The second read of each Q_k element comes from cache; per-thread order and block sums are those of
// update_kernel followed by multidot_kernel, so the results are identical.
template <int KT>
__global__ void __launch_bounds__(KRYLOV_THREADS)
update_multidot_kernel(const double2 *__restrict__ Q, size_t n, size_t qs, int kc, const double2 *__restrict__ z,
                       double2 *__restrict__ v, double2 *__restrict__ partial, int ld, const KrylovStatus *st)
{
    const int inst = blockIdx.y;
    Q += inst * n; v += inst * n; z += (size_t)inst * ld; partial += (size_t)inst * gridDim.x * ld;
    if (st) st += inst;
    if (st && st->done) return;
    __shared__ double2 zs[KT];
    for (int k = threadIdx.x; k < kc; k += blockDim.x) zs[k] = z[k];
    __syncthreads();
    double2 acc[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) acc[k] = mk<double>(0, 0);
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        double2 x = v[p];
#pragma unroll
        for (int k = 0; k < KT; ++k)
            if (k < kc) x = cfma<double>(mk<double>(-zs[k].x, -zs[k].y), Q[(size_t)k * qs + p], x);
        v[p] = x;
#pragma unroll
        for (int k = 0; k < KT; ++k)
            if (k < kc) acc[k] = cfma_conj<double>(Q[(size_t)k * qs + p], x, acc[k]);
    }
    __shared__ double2 res[KT];
    block_sum<KT>(acc, res);
    __syncthreads();
    if (threadIdx.x < kc) partial[(size_t)blockIdx.x * ld + threadIdx.x] = res[threadIdx.x];
}

// per-block |v|^2
__global__ void __launch_bounds__(KRYLOV_THREADS)
norm_kernel(const double2 *__restrict__ v, size_t n, double *__restrict__ norm_partial)
{
    v += blockIdx.y * n; norm_partial += (size_t)blockIdx.y * gridDim.x;
    double nrm = 0;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        nrm += cabs2<double>(v[p]);
    __shared__ double red[KRYLOV_THREADS / 32];
    const double s = warp_sum(nrm);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < KRYLOV_THREADS / 32; ++w) t += red[w];
        norm_partial[blockIdx.x] = t;
    }
}

// h = sqrt(sum of partials) -> H[j+1, j], status.hnext, happy flag (h < 1e-13).
__global__ void finish_norm_kernel(const double *__restrict__ norm_partial, int nb, double2 *hsub, size_t hs,
                                   KrylovStatus *st, double happy_below)
{
    const int inst = blockIdx.x;
    norm_partial += (size_t)inst * nb; hsub += inst * hs; st += inst;
    if (st->done) return;
    const double s = warp_fixed_sum(norm_partial, nb, 1);
    if (threadIdx.x != 0) return;
    const double h = sqrt(s);
    *hsub = mk<double>(h, 0);
    st->hnext = h;
    st->happy = h < happy_below;
}

// y = s * x with s = 1 / status.hnext (skipped once the solve is done)
__global__ void __launch_bounds__(KRYLOV_THREADS)
normalize_kernel(const double2 *x, double2 *y, size_t n, const KrylovStatus *st)
{
    x += blockIdx.y * n; y += blockIdx.y * n; st += blockIdx.y;
    if (st->done) return;
    const double s = 1.0 / st->hnext;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        y[p] = cscale<double>(s, x[p]);
}

// start: beta = ||x||, Q_0 = x / beta (reads beta from the reduced norm)
__global__ void start_kernel(const double *__restrict__ norm_partial, int nb, KrylovStatus *st)
{
    norm_partial += (size_t)blockIdx.x * nb; st += blockIdx.x;
    const double s = warp_fixed_sum(norm_partial, nb, 1);
    if (threadIdx.x != 0) return;
    memset(st, 0, sizeof(KrylovStatus));
    st->beta = sqrt(s);
    st->hnext = st->beta;
    if (st->beta == 0) { st->done = 1; st->converged = 1; st->m = 0; }
}

// y = sum_{k < m} Q_k c_k with m taken from the status word (or from `mfix` >= 0).  With
// the status word (mfix < 0), y is left untouched unless the solve converged.
__global__ void __launch_bounds__(KRYLOV_THREADS)
combine_kernel(const double2 *__restrict__ Q, size_t n, size_t qs, const double2 *__restrict__ c, int ld,
               double2 *__restrict__ y, const KrylovStatus *st, int mfix, int accumulate)
{
    const int inst = blockIdx.y;
    Q += inst * n; c += (size_t)inst * ld; y += inst * n; st += inst;
    if (mfix < 0 && (st->failed || !st->converged)) return;
    const int m = mfix >= 0 ? mfix : st->m;
    __shared__ double2 cs[KRYLOV_MAXDIM];
    for (int k = threadIdx.x; k < m; k += blockDim.x) cs[k] = c[k];
    __syncthreads();
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        double2 acc = accumulate ? y[p] : mk<double>(0, 0);
        for (int k = 0; k < m; ++k) acc = cfma<double>(cs[k], Q[(size_t)k * qs + p], acc);
        y[p] = acc;
    }
}

// ---------------------------------------------------------------------------------
// Small dense complex matrices on one CTA (column-major, leading dimension m).
// ---------------------------------------------------------------------------------
__device__ void mat_mul(const double2 *A, const double2 *B, double2 *C, int m)
{
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
        const int i = idx % m, j = idx / m;
        double2 s = mk<double>(0, 0);
        for (int k = 0; k < m; ++k) s = cfma<double>(A[i + k * m], B[k + j * m], s);
        C[idx] = s;
    }
    __syncthreads();
}

// C = a*A + b*B + c*Cm + d*I   (real coefficients)
__device__ void mat_lin(double2 *out, double a, const double2 *A, double b, const double2 *B, double c,
                        const double2 *Cm, double d, int m)
{
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
        double2 s = cscale<double>(a, A[idx]);
        if (B) s = rfma<double>(b, B[idx], s);
        if (Cm) s = rfma<double>(c, Cm[idx], s);
        if (idx % m == idx / m) s.x += d;
        out[idx] = s;
    }
    __syncthreads();
}

// Solve A X = B in place (B overwritten by X), Gaussian elimination with partial pivoting.
__device__ void lu_solve(double2 *A, double2 *B, int m, int nrhs)
{
    __shared__ int piv;
    for (int k = 0; k < m; ++k) {
        if (threadIdx.x == 0) {
            int best = k;
            double bv = cabs2<double>(A[k + k * m]);
            for (int i = k + 1; i < m; ++i) {
                const double v = cabs2<double>(A[i + k * m]);
                if (v > bv) { bv = v; best = i; }
            }
            piv = best;
        }
        __syncthreads();
        const int p = piv;
        if (p != k) {
            for (int j = threadIdx.x; j < m; j += blockDim.x) {
                const double2 t = A[k + j * m]; A[k + j * m] = A[p + j * m]; A[p + j * m] = t;
            }
            for (int j = threadIdx.x; j < nrhs; j += blockDim.x) {
                const double2 t = B[k + j * m]; B[k + j * m] = B[p + j * m]; B[p + j * m] = t;
            }
        }
        __syncthreads();
        const double2 d = A[k + k * m];
        const double dd = cabs2<double>(d);
        const double2 inv = mk<double>(d.x / dd, -d.y / dd);
        // eliminate rows below k
        for (int idx = threadIdx.x; idx < (m - k - 1) * (m - k + nrhs); idx += blockDim.x) {
            const int i = k + 1 + idx % (m - k - 1);
            const int jj = idx / (m - k - 1);
            const double2 f = cmul<double>(A[i + k * m], inv);
            if (jj < m - k - 1) {
                const int j = k + 1 + jj;
                A[i + j * m] = csub<double>(A[i + j * m], cmul<double>(f, A[k + j * m]));
            } else {
                const int j = jj - (m - k - 1);
                B[i + j * m] = csub<double>(B[i + j * m], cmul<double>(f, B[k + j * m]));
            }
        }
        __syncthreads();
        for (int i = k + 1 + threadIdx.x; i < m; i += blockDim.x) A[i + k * m] = mk<double>(0, 0);
        __syncthreads();
    }
    // back substitution, one right-hand side per thread group
    for (int j = threadIdx.x; j < nrhs; j += blockDim.x) {
        for (int i = m - 1; i >= 0; --i) {
            double2 s = B[i + j * m];
            for (int k = i + 1; k < m; ++k) s = csub<double>(s, cmul<double>(A[i + k * m], B[k + j * m]));
            const double2 d = A[i + i * m];
            const double dd = cabs2<double>(d);
            B[i + j * m] = mk<double>((s.x * d.x + s.y * d.y) / dd, (s.y * d.x - s.x * d.y) / dd);
        }
    }
    __syncthreads();
}

// expm(A) for a small complex matrix: scaling and squaring with the [13/13] Pade
// approximant (N. J. Higham, SIAM J. Matrix Anal. Appl. 26 (2005) 1179-1193).
// A is overwritten; the result is left in R.  work holds 6 m x m matrices.
__device__ void expm_pade13(double2 *A, double2 *R, double2 *work, int m)
{
    const double b[14] = {64764752532480000., 32382376266240000., 7771770303897600., 1187353796428800.,
                          129060195264000., 10559470521600., 670442572800., 33522128640., 1323241920.,
                          40840800., 960960., 16380., 182., 1.};
    const double theta13 = 5.371920351148152;
    __shared__ int s_shared;
    if (threadIdx.x == 0) {
        double norm1 = 0;     // max column sum
        for (int j = 0; j < m; ++j) {
            double c = 0;
            for (int i = 0; i < m; ++i) c += sqrt(cabs2<double>(A[i + j * m]));
            norm1 = fmax(norm1, c);
        }
        int s = 0;
        if (norm1 > theta13) s = (int)ceil(log2(norm1 / theta13));
        s_shared = s;
    }
    __syncthreads();
    const int s = s_shared;
    const double scale = ldexp(1.0, -s);
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) A[idx] = cscale<double>(scale, A[idx]);
    __syncthreads();
    double2 *A2 = work, *A4 = work + m * m, *A6 = work + 2 * m * m, *T = work + 3 * m * m, *U = work + 4 * m * m,
            *V = work + 5 * m * m;
    mat_mul(A, A, A2, m);
    mat_mul(A2, A2, A4, m);
    mat_mul(A4, A2, A6, m);
    // U = A [A6 (b13 A6 + b11 A4 + b9 A2) + b7 A6 + b5 A4 + b3 A2 + b1 I]
    mat_lin(T, b[13], A6, b[11], A4, b[9], A2, 0.0, m);
    mat_mul(A6, T, U, m);
    mat_lin(T, 1.0, U, b[7], A6, b[5], A4, b[1], m);
    mat_lin(T, 1.0, T, b[3], A2, 0.0, nullptr, 0.0, m);
    mat_mul(A, T, U, m);
    // V = A6 (b12 A6 + b10 A4 + b8 A2) + b6 A6 + b4 A4 + b2 A2 + b0 I
    mat_lin(T, b[12], A6, b[10], A4, b[8], A2, 0.0, m);
    mat_mul(A6, T, V, m);
    mat_lin(V, 1.0, V, b[6], A6, b[4], A4, b[0], m);
    mat_lin(V, 1.0, V, b[2], A2, 0.0, nullptr, 0.0, m);
    // (V - U) R = (V + U)
    mat_lin(T, 1.0, V, -1.0, U, 0.0, nullptr, 0.0, m);
    mat_lin(R, 1.0, V, 1.0, U, 0.0, nullptr, 0.0, m);
    lu_solve(T, R, m, m);
    for (int k = 0; k < s; ++k) {
        mat_mul(R, R, T, m);
        mat_lin(R, 1.0, T, 0.0, nullptr, 0.0, nullptr, 0.0, m);
    }
}

// Arnoldi check at iteration j (python/propagate.py:28-38) by the whole calling block: on
// happy breakdown or at j >= 3 with (j+1) % 4 == 0 or j+1 == maxdim, form
// c = expm(-i dt H_m)[:, 0] beta and err = |dt h_{m+1,m} c_{m-1}|; accept if happy or
// err < tol.  H, coef, work and st are this instance's slices.
__device__ __noinline__ void arnoldi_check_block(const double2 *__restrict__ H, int ld, int j, int maxdim, double dt, double tol,
                                    double2 *__restrict__ coef, double2 *__restrict__ work, KrylovStatus *st)
{
    if (tol < 0) return;   // a GMRES iteration: the sweeps without the exponential's check
    const int m = j + 1;
    const bool happy = st->happy;
    const bool check = happy || (j >= 3 && ((j + 1) % 4 == 0 || j + 1 == maxdim));
    if (!check) return;
    // the 8 small matrices of the exponential in shared memory when they fit (m <= 16)
    constexpr int SMALL = 16;
    __shared__ double2 small[8 * SMALL * SMALL];
    if (m <= SMALL) work = small;
    double2 *A = work, *R = work + m * m, *scratch = work + 2 * m * m;
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
        const int r = idx % m, c = idx / m;
        const double2 h = H[r + c * ld];
        A[idx] = mk<double>(dt * h.y, -dt * h.x);   // -i dt H
    }
    __syncthreads();
    expm_pade13(A, R, scratch, m);
    if (threadIdx.x == 0) {
        const double beta = st->beta;
        for (int k = 0; k < m; ++k) coef[k] = cscale<double>(beta, R[k]);
        const double err = fabs(dt) * st->hnext * sqrt(cabs2<double>(coef[m - 1]));
        st->estimate = err;
        if (happy || err < tol) {
            st->done = 1; st->converged = 1; st->m = m;
        } else if (j + 1 == maxdim) {
            st->done = 1; st->failed = 1; st->m = m;
        }
    }
}

__global__ void __launch_bounds__(512)
arnoldi_check_kernel(const double2 *__restrict__ H, int ld, size_t hs, int j, int maxdim, double dt, double tol,
                     double2 *__restrict__ coef, double2 *__restrict__ work, size_t ws, KrylovStatus *st)
{
    const int inst = blockIdx.x;
    H += inst * hs; coef += (size_t)inst * ld; work += inst * ws; st += inst;
    if (st->done) return;
    arnoldi_check_block(H, ld, j, maxdim, dt, tol, coef, work, st);
}

// ---------------------------------------------------------------------------------
// One Arnoldi iteration in three sweeps (kc = j + 1 <= KRYLOV_FUSED basis vectors):
//   project:  z = Q^H v                                    (H[:, j] += z)
//   reorth:   v' = v - Q z; z' = Q^H v'; |v'|^2             (H[:, j] += z')
//             h = sqrt(|v'|^2 - |z'|^2) = |v' - Q z'|        (H[j+1, j], happy flag)
//             + the Arnoldi check on the same block
//   next:     Q_{j+1} = (v' - Q z') / h                       (skipped once done)
// Each reduction ends in the last block to finish (ticket counter): it sums the block
// partials in a fixed order (lane l adds blocks l, l+32, ... in sequence, then a butterfly),
// so results do not depend on timing.  |v'' |^2 = |v'|^2 - |z'|^2 holds because Q has
// orthonormal columns; after the first sweep |z'| is at rounding level, so the subtraction
// loses nothing.
// ---------------------------------------------------------------------------------
constexpr int KRYLOV_LANE_LOADS = (KRYLOV_BLOCKS + 31) / 32;

// Fixed-order sum of nb <= KRYLOV_BLOCKS partials p[b * ld] by one warp (all loads issued
// before the adds; L1 bypassed, the partials come from other SMs).
__device__ __forceinline__ double2 ordered_partial_sum(const double2 *p, int nb, int ld)
{
    const int lane = threadIdx.x & 31;
    double2 v[KRYLOV_LANE_LOADS];
#pragma unroll
    for (int i = 0; i < KRYLOV_LANE_LOADS; ++i) {
        const int b = lane + 32 * i;
        v[i] = b < nb ? __ldcg(p + (size_t)b * ld) : mk<double>(0, 0);
    }
    double2 s = mk<double>(0, 0);
#pragma unroll
    for (int i = 0; i < KRYLOV_LANE_LOADS; ++i) s = cadd<double>(s, v[i]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, off);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, off);
    }
    return s;
}

// Load that the compiler may neither merge with an earlier load of the same address nor
// move: a value read again instead of being held in a register.
__device__ __forceinline__ double2 reload(const double2 *p)
{
    double2 v;
    asm volatile("ld.global.ca.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}

// Every thread has written its partials; returns true in the last block to arrive (which
// then sees every block's partials).  No waiting: the other blocks just return.
__device__ __forceinline__ bool arrive_last(unsigned int *ticket)
{
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (s_last) __threadfence();
    return s_last;
}

// project: partials of conj(Q_k) v, last block -> z, H[:, j] += z.  With src32, v is first
// filled from the complex64 operator result (mixed precision).
template <int KT>
__global__ void __launch_bounds__(KRYLOV_THREADS)
arnoldi_project_kernel(const double2 *__restrict__ Q, size_t n, size_t qs, int kc, double2 *__restrict__ v,
                       const float2 *__restrict__ src32, double2 *__restrict__ partial, int ld,
                       unsigned int *__restrict__ ticket, double2 *__restrict__ z, double2 *__restrict__ H, size_t hs,
                       int j, const KrylovStatus *st)
{
    const int inst = blockIdx.y;
    Q += inst * n; v += inst * n; partial += (size_t)inst * gridDim.x * ld; st += inst;
    z += (size_t)inst * ld; H += inst * hs; ticket += inst;
    if (src32) src32 += inst * n;
    if (st->done) return;
    double2 acc[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) acc[k] = mk<double>(0, 0);
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        double2 x;
        if (src32) {
            const float2 f = src32[p];
            x = mk<double>((double)f.x, (double)f.y);
            v[p] = x;
        } else {
            x = v[p];
        }
#pragma unroll
        for (int k = 0; k < KT; ++k)
            if (k < kc) acc[k] = cfma_conj<double>(Q[(size_t)k * qs + p], x, acc[k]);
    }
    __shared__ double2 res[KT];
    block_sum<KT>(acc, res);
    __syncthreads();
    if (threadIdx.x < kc) partial[(size_t)blockIdx.x * ld + threadIdx.x] = res[threadIdx.x];
    if (!arrive_last(ticket)) return;
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int k = warp; k < kc; k += nwarps) {
        const double2 s = ordered_partial_sum(partial + k, gridDim.x, ld);
        if ((threadIdx.x & 31) == 0) {
            z[k] = s;
            H[k + (size_t)j * ld] = cadd<double>(H[k + (size_t)j * ld], s);
        }
    }
    if (threadIdx.x == 0) *ticket = 0;
}

// reorth: v' = v - Q z written; partials of conj(Q_k) v' and |v'|^2 (column kc); last
// block -> z' (into z), H[:, j] += z', h, happy flag, then the Arnoldi check.
template <int KT>
__global__ void __launch_bounds__(KRYLOV_THREADS, 3)
arnoldi_reorth_kernel(const double2 *__restrict__ Q, size_t n, size_t qs, int kc, double2 *__restrict__ z,
                      double2 *__restrict__ v, double2 *__restrict__ partial, int ld, unsigned int *__restrict__ ticket,
                      double2 *__restrict__ H, size_t hs, int j, int maxdim, double dt, double tol,
                      double2 *__restrict__ coef, double2 *__restrict__ work, size_t ws, KrylovStatus *st,
                      double happy_below)
{
    const int inst = blockIdx.y;
    Q += inst * n; v += inst * n; partial += (size_t)inst * gridDim.x * ld; st += inst;
    z += (size_t)inst * ld; H += inst * hs; ticket += inst; coef += (size_t)inst * ld; work += inst * ws;
    if (st->done) return;
    __shared__ double2 zs[KT];
    for (int k = threadIdx.x; k < kc; k += blockDim.x) zs[k] = z[k];
    __syncthreads();
    double2 acc[KT + 1];
#pragma unroll
    for (int k = 0; k <= KT; ++k) acc[k] = mk<double>(0, 0);
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        double2 x = v[p];
#pragma unroll
        for (int k = 0; k < KT; ++k)
            if (k < kc) x = cfma<double>(mk<double>(-zs[k].x, -zs[k].y), Q[(size_t)k * qs + p], x);
        v[p] = x;
        // second use of the basis elements: read again (from L1) rather than kept in
        // registers, so that the kernel keeps its occupancy
#pragma unroll
        for (int k = 0; k < KT; ++k)
            if (k < kc) acc[k] = cfma_conj<double>(reload(Q + (size_t)k * qs + p), x, acc[k]);
        acc[KT].x += cabs2<double>(x);
    }
    __shared__ double2 res[KT + 1];
    block_sum<KT + 1>(acc, res);
    __syncthreads();
    if (threadIdx.x < kc) partial[(size_t)blockIdx.x * ld + threadIdx.x] = res[threadIdx.x];
    if (threadIdx.x == kc) partial[(size_t)blockIdx.x * ld + kc] = res[KT];
    if (!arrive_last(ticket)) return;
    __shared__ double2 tot[KT + 1];
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int k = warp; k <= kc; k += nwarps) {
        const double2 s = ordered_partial_sum(partial + k, gridDim.x, ld);
        if ((threadIdx.x & 31) == 0) tot[k] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double h2 = tot[kc].x;
        for (int k = 0; k < kc; ++k) {
            z[k] = tot[k];
            H[k + (size_t)j * ld] = cadd<double>(H[k + (size_t)j * ld], tot[k]);
            h2 -= cabs2<double>(tot[k]);
        }
        const double h = sqrt(fmax(h2, 0.0));
        H[j + 1 + (size_t)j * ld] = mk<double>(h, 0);
        st->hnext = h;
        st->happy = h < happy_below;
        *ticket = 0;
    }
    __syncthreads();
    arnoldi_check_block(H, ld, j, maxdim, dt, tol, coef, work, st);
}

// next: Q_{j+1} = (v' - Q z') / h in place (and its complex64 copy for the next
// mixed-precision apply); nothing once the solve is done.
__global__ void __launch_bounds__(KRYLOV_THREADS)
arnoldi_next_kernel(const double2 *__restrict__ Q, size_t n, size_t qs, int kc, const double2 *__restrict__ z, int ld,
                    double2 *__restrict__ v, float2 *__restrict__ out32, const KrylovStatus *st)
{
    const int inst = blockIdx.y;
    Q += inst * n; v += inst * n; z += (size_t)inst * ld; st += inst;
    if (out32) out32 += inst * n;
    if (st->done) return;
    __shared__ double2 zs[KRYLOV_MAXDIM + 1];
    for (int k = threadIdx.x; k < kc; k += blockDim.x) zs[k] = z[k];
    __syncthreads();
    const double s = 1.0 / st->hnext;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
        double2 x = v[p];
        for (int k = 0; k < kc; ++k) x = cfma<double>(mk<double>(-zs[k].x, -zs[k].y), Q[(size_t)k * qs + p], x);
        x = cscale<double>(s, x);
        v[p] = x;
        if (out32) out32[p] = make_float2((float)x.x, (float)x.y);
    }
}

}  // namespace he

// =====================================================================================
// Host side
// =====================================================================================
using namespace he;

he_krylov::~he_krylov()
{
    cudaFree(Q); cudaFree(Z); cudaFree(H); cudaFree(partial); cudaFree(z); cudaFree(coef); cudaFree(work);
    cudaFree(norm_partial); cudaFree(status); cudaFree(ticket); cudaFree(s32[0]); cudaFree(s32[1]);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (capture_stream) cudaStreamDestroy(capture_stream);
    if (host_status) cudaFreeHost(host_status);
    he_gmres_buffers_free(gmres);
}

namespace {
int krylov_create(he_krylov **out, long long n, int maxdim, int flexible, int count)
{
    if (!out) return he_fail(HE_ERR_ARG, "null handle pointer", __FILE__, __LINE__);
    *out = nullptr;
    if (n < 1 || maxdim < 1 || maxdim > KRYLOV_MAXDIM)
        return he_fail(HE_ERR_ARG, "Krylov dimension must be in [1, 64] and n >= 1", __FILE__, __LINE__);
    if (count < 1 || count > HE_BATCH_MAX) return he_fail(HE_ERR_ARG, "batch count must be in [1, 64]", __FILE__, __LINE__);
    he_krylov *k = new he_krylov();
    k->n = (size_t)n; k->maxdim = maxdim; k->flexible = flexible; k->count = count;
    cudaError_t e = cudaGetDevice(&k->device);
    // one instance: KRYLOV_BLOCKS CTAs; a batch: about four CTAs per SM over all instances
    // (the sweeps of a batch stream from HBM and need the warps to keep enough loads in flight)
    if (count > 1)
        k->blocks = std::min(KRYLOV_BLOCKS, std::max(8, 4 * sm_count(k->device) / count));
    const size_t ld = maxdim + 1, c = count;
    if (e == cudaSuccess) e = cudaMalloc(&k->Q, ld * c * k->n * sizeof(double2));
    if (e == cudaSuccess && flexible) e = cudaMalloc(&k->Z, (size_t)maxdim * c * k->n * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&k->H, c * ld * maxdim * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&k->partial, c * KRYLOV_BLOCKS * ld * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&k->z, c * ld * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&k->coef, c * ld * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&k->work, c * 8 * ld * ld * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&k->norm_partial, c * KRYLOV_BLOCKS * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&k->status, c * sizeof(KrylovStatus));
    if (e == cudaSuccess) e = cudaMalloc(&k->ticket, c * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(k->ticket, 0, c * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost(&k->host_status, c * sizeof(KrylovStatus));
    if (e != cudaSuccess) {
        he_set_error(cudaGetErrorString(e), __FILE__, __LINE__);
        delete k;
        return HE_ERR_CUDA;
    }
    *out = k;
    return HE_OK;
}
}  // namespace

extern "C" int he_krylov_create(he_krylov **out, long long n, int maxdim, int flexible)
{
    return krylov_create(out, n, maxdim, flexible, 1);
}

extern "C" int he_krylov_create_batched(he_krylov **out, long long n, int maxdim, int count)
{
    return krylov_create(out, n, maxdim, 0, count);
}

extern "C" int he_krylov_set_graphs(he_krylov *k, int enable)
{
    if (!k) return he_fail(HE_ERR_ARG, "null handle", __FILE__, __LINE__);
    k->graphs = enable != 0;
    k->graph_key = 0;
    return HE_OK;
}

// Solves whose graph capture failed and were enqueued directly (total), and whether the
// workspace still captures (graphs are turned off after repeated failures in a row).
extern "C" int he_krylov_capture_fallbacks(he_krylov *k, int *fallbacks, int *graphs_on)
{
    if (!k) return he_fail(HE_ERR_ARG, "null handle", __FILE__, __LINE__);
    if (fallbacks) *fallbacks = k->capture_fallbacks;
    if (graphs_on) *graphs_on = k->graphs ? 1 : 0;
    return HE_OK;
}

extern "C" int he_krylov_destroy(he_krylov *k)
{
    delete k;
    return HE_OK;
}

extern "C" int he_krylov_vector(he_krylov *k, int which, int j, void **ptr)
{
    if (!k || !ptr) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (which == 0 && j >= 0 && j <= k->maxdim) *ptr = k->Q + (size_t)j * k->qs();
    else if (which == 1 && k->Z && j >= 0 && j < k->maxdim) *ptr = k->Z + (size_t)j * k->n;
    else return he_fail(HE_ERR_ARG, "basis index out of range", __FILE__, __LINE__);
    return HE_OK;
}

namespace he {

static const dim3 kBlock(KRYLOV_THREADS);
inline dim3 bgrid(const he_krylov *k) { return dim3(k->kb(), k->count); }   // every instance

int krylov_multidot(he_krylov *k, int kc, const double2 *v, double2 *hcol, cudaStream_t s, const KrylovStatus *st,
                    const double2 *basis)
{
    const int ld = k->maxdim + 1;
    for (int k0 = 0; k0 < kc; k0 += KRYLOV_TILE) {
        const int t = kc - k0 < KRYLOV_TILE ? kc - k0 : KRYLOV_TILE;
        multidot_kernel<KRYLOV_TILE><<<bgrid(k), kBlock, 0, s>>>(basis, k->n, k->qs(), k0, t, v, k->partial, ld, st);
    }
    reduce_partials_kernel<<<k->count, 32 * std::max(1, std::min(kc, 16)), 0, s>>>(k->partial, k->kb(), ld, kc, k->z,
                                                                                  hcol, k->hs(), st);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

// CGS2 of v against basis[0..kc): twice (projection, update), H column += projections,
// then h = ||v|| into *hsub and the status word.
int krylov_cgs2(he_krylov *k, int kc, double2 *v, double2 *hcol, double2 *hsub, cudaStream_t s, double happy_below)
{
    int rc;
    if (kc <= KRYLOV_FUSED) {   // three sweeps: project, update + project, update + norm
        const int ld = k->maxdim + 1;
        if ((rc = krylov_multidot(k, kc, v, hcol, s, k->status, k->Q))) return rc;
        update_multidot_kernel<KRYLOV_FUSED><<<bgrid(k), kBlock, 0, s>>>(k->Q, k->n, k->qs(), kc, k->z, v, k->partial, ld,
                                                                        k->status);
        reduce_partials_kernel<<<k->count, 32 * std::max(1, std::min(kc, 16)), 0, s>>>(k->partial, k->kb(), ld, kc,
                                                                                      k->z, hcol, k->hs(), k->status);
        update_kernel<<<bgrid(k), kBlock, 0, s>>>(k->Q, k->n, k->qs(), kc, k->z, ld, v, k->norm_partial, k->status);
    } else {
        for (int rep = 0; rep < 2; ++rep) {
            if ((rc = krylov_multidot(k, kc, v, hcol, s, k->status, k->Q))) return rc;
            update_kernel<<<bgrid(k), kBlock, 0, s>>>(k->Q, k->n, k->qs(), kc, k->z, k->maxdim + 1, v,
                                                      rep == 1 ? k->norm_partial : nullptr, k->status);
        }
    }
    finish_norm_kernel<<<k->count, 32, 0, s>>>(k->norm_partial, k->kb(), hsub, k->hs(), k->status, happy_below);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

int krylov_start(he_krylov *k, const double2 *x, cudaStream_t s)
{
    norm_kernel<<<bgrid(k), kBlock, 0, s>>>(x, k->n, k->norm_partial);
    start_kernel<<<k->count, 32, 0, s>>>(k->norm_partial, k->kb(), k->status);
    normalize_kernel<<<bgrid(k), kBlock, 0, s>>>(x, k->Q, k->n, k->status);
    HE_CUDA_TRY(cudaMemsetAsync(k->H, 0, sizeof(double2) * k->hs() * k->count, s));
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

int krylov_read_status(he_krylov *k, cudaStream_t s)
{
    HE_CUDA_TRY(cudaMemcpyAsync(k->host_status, k->status, sizeof(KrylovStatus) * k->count, cudaMemcpyDeviceToHost, s));
    HE_CUDA_TRY(cudaStreamSynchronize(s));
    return HE_OK;
}

}  // namespace he

// Arnoldi steps for an operator applied by the caller:
//   start(x) -> beta; for j: caller writes H Q_j into vector j+1; orthogonalize(j);
//   check(j) -> done?; when done: combine(y).
extern "C" int he_krylov_start(he_krylov *k, const void *x, double *beta, void *stream)
{
    if (!k || !x) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    int rc = krylov_start(k, static_cast<const double2 *>(x), s);
    if (!rc) rc = krylov_read_status(k, s);
    if (!rc && beta) *beta = k->host_status->beta;
    return rc;
}

extern "C" int he_krylov_orthogonalize(he_krylov *k, int j, void *stream)
{
    if (!k || j < 0 || j >= k->maxdim) return he_fail(HE_ERR_ARG, "bad Arnoldi index", __FILE__, __LINE__);
    const int ld = k->maxdim + 1;
    double2 *v = k->Q + (size_t)(j + 1) * k->qs();
    return krylov_cgs2(k, j + 1, v, k->H + (size_t)j * ld, k->H + (size_t)j * ld + j + 1,
                       static_cast<cudaStream_t>(stream), 1e-13);
}

// Device-side check at iteration j, normalization of vector j+1 when not done.
// sync != 0 reads the status back (done, m, estimate) and blocks the host.
extern "C" int he_expv_check(he_krylov *k, int j, int maxdim, double dt, double tol, int sync, int *done, int *m,
                             double *estimate, void *stream)
{
    if (!k || maxdim < 1 || maxdim > k->maxdim || j < 0 || j >= maxdim)
        return he_fail(HE_ERR_ARG, "bad Arnoldi index", __FILE__, __LINE__);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    arnoldi_check_kernel<<<k->count, 512, 0, s>>>(k->H, k->maxdim + 1, k->hs(), j, maxdim, dt, tol, k->coef, k->work,
                                                  k->ws(), k->status);
    if (j + 1 < maxdim)
        normalize_kernel<<<bgrid(k), kBlock, 0, s>>>(k->Q + (size_t)(j + 1) * k->qs(), k->Q + (size_t)(j + 1) * k->qs(), k->n,
                                                  k->status);
    HE_CUDA_TRY(cudaGetLastError());
    if (sync) {
        int rc = krylov_read_status(k, s);
        if (rc) return rc;
        if (done) *done = k->host_status->done;
        if (m) *m = k->host_status->m;
        if (estimate) *estimate = k->host_status->estimate;
        if (k->host_status->failed) return he_fail(HE_ERR_NOCONV, "Arnoldi did not converge", __FILE__, __LINE__);
    }
    return HE_OK;
}

// Q_j /= h_{j,j-1} from the status word (the norm of the last orthogonalisation), on the
// device: the GMRES driver reads the Hessenberg only at its check points.
extern "C" int he_krylov_normalize(he_krylov *k, int j, void *stream)
{
    if (!k || j < 1 || j > k->maxdim) return he_fail(HE_ERR_ARG, "bad basis index", __FILE__, __LINE__);
    double2 *q = k->Q + (size_t)j * k->qs();
    normalize_kernel<<<bgrid(k), kBlock, 0, static_cast<cudaStream_t>(stream)>>>(q, q, k->n, k->status);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

extern "C" int he_krylov_combine(he_krylov *k, int m, void *y, void *stream)
{
    if (!k || !y || m > k->maxdim) return he_fail(HE_ERR_ARG, "bad combination", __FILE__, __LINE__);
    combine_kernel<<<bgrid(k), kBlock, 0, static_cast<cudaStream_t>(stream)>>>(k->Q, k->n, k->qs(), k->coef, k->maxdim + 1,
                                                                                static_cast<double2 *>(y), k->status, m, 0);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

// Fused Arnoldi exponential action y = exp(-i dt H(field)) x with the device operator.
// Host syncs only at the reference's check points (m = 4, 8, ..., maxdim).
namespace {
__global__ void krylov_to_c64(size_t n, const double2 *x, float2 *y)
{
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        y[p] = make_float2((float)x[p].x, (float)x[p].y);
}
__global__ void krylov_to_c128(size_t n, const float2 *x, double2 *y)
{
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
        y[p] = make_double2((double)x[p].x, (double)x[p].y);
}

// Grid of a fused sweep: one instance keeps KRYLOV_BLOCKS CTAs; a batch gets as many CTAs
// per instance as fill the SMs in one wave at the kernel's own occupancy (the sweeps of a
// batch stream from HBM), at most KRYLOV_BLOCKS (the size of the partial-sum slices).
dim3 sweep_grid(const he_krylov *k, const void *kernel)
{
    if (k->count == 1) return bgrid(k);
    const int per_sm = resident_ctas(kernel, KRYLOV_THREADS, 0);
    const int blocks = std::min(KRYLOV_BLOCKS, std::max(8, per_sm * sm_count(k->device) / k->count));
    return dim3(blocks, k->count);
}

// project + reorth(+ check) sweeps of one fused Arnoldi iteration, with the register tile
// sized to the basis (4, 8, 12 or 16 vectors).
template <int KT>
void launch_fused_sweeps(he_krylov *k, int kc, double2 *v, const float2 *src32, int j, int maxdim, double dt,
                         double tol, cudaStream_t s, double happy_below)
{
    const int ld = k->maxdim + 1;
    arnoldi_project_kernel<KT><<<sweep_grid(k, reinterpret_cast<const void *>(arnoldi_project_kernel<KT>)), kBlock, 0, s>>>(k->Q, k->n, k->qs(), kc, v, src32, k->partial, ld, k->ticket,
                                                          k->z, k->H, k->hs(), j, k->status);
    arnoldi_reorth_kernel<KT><<<sweep_grid(k, reinterpret_cast<const void *>(arnoldi_reorth_kernel<KT>)), kBlock, 0, s>>>(
        k->Q, k->n, k->qs(), kc, k->z, v, k->partial, ld, k->ticket,
                                                         k->H, k->hs(), j, maxdim, dt, tol, k->coef, k->work, k->ws(),
                                                         k->status, happy_below);
}

int fused_sweeps(he_krylov *k, int kc, double2 *v, const float2 *src32, int j, int maxdim, double dt, double tol,
                 cudaStream_t s, double happy_below = 1e-13)
{
    if (kc <= 4) launch_fused_sweeps<4>(k, kc, v, src32, j, maxdim, dt, tol, s, happy_below);
    else if (kc <= 8) launch_fused_sweeps<8>(k, kc, v, src32, j, maxdim, dt, tol, s, happy_below);
    else if (kc <= 12) launch_fused_sweeps<12>(k, kc, v, src32, j, maxdim, dt, tol, s, happy_below);
    else launch_fused_sweeps<KRYLOV_FUSED>(k, kc, v, src32, j, maxdim, dt, tol, s, happy_below);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

// y_b = exp(-i dt H(fields_b)) x_b for every instance of the workspace.  precision HE_C64:
// H·psi in complex64 (the basis, CGS2, the Hessenberg exponential and the error estimate
// stay complex128).  Per-instance dimensions, estimates and convergence go to the optional
// arrays; the status is HE_ERR_NOCONV when any instance did not converge (its y_b is left
// as it was).
// Every kernel of one Arnoldi solve, enqueued on s without waiting on the device: the check
// decides convergence at the reference's check points on the device and sets the status
// word, after which every Krylov kernel returns at once.  (x = 0 gives beta = 0: done at
// once with m = 0, and the combination writes y = 0 = x.)
// Iterations j0 .. j1-1 of the solve (j0 = 0 starts it), then y = Q c if it has converged.
// The kernels see the solve's maxdim whatever the segment, so a solve enqueued in segments
// runs exactly the launches of one enqueued whole.
// direction != null: the field-derivative block operator of he_expv_field_derivative on
// x = [u; w] (k->n = 2 N): B [u; w] = [H u + (direction . d) w; H w], one batched apply of the
// two halves and the dipole coupling added to the upper half.
int enqueue_expv(he_krylov *k, he_handle op, const void *x, void *y, const double *fields, int velocity, double dt,
                 double tol, int maxdim, cudaStream_t s, int precision, const double *direction, int j0, int j1)
{
    const size_t total = k->qs();   // one basis vector of every instance
    int rc = HE_OK;
    if (j0 == 0) {
        if ((rc = krylov_start(k, static_cast<const double2 *>(x), s))) return rc;
        HE_CUDA_TRY(cudaMemsetAsync(k->ticket, 0, sizeof(unsigned int) * k->count, s));
    }
    const int ld = k->maxdim + 1;
    const dim3 cgrid(std::min<size_t>(KRYLOV_BLOCKS * (size_t)k->count, 4096));
    const bool mixed = precision == HE_C64;
    // a single solve's applies return at once after its convergence
    const int *gate = k->count == 1 ? &k->status->done : nullptr;
    // s32[0] holds the complex64 copy of Q_j (written by the previous iteration when it was fused)
    bool have32 = mixed && j0 >= 1 && j0 <= KRYLOV_FUSED;
    for (int j = j0; j < j1; ++j) {
        double2 *qj = k->Q + (size_t)j * total, *v = k->Q + (size_t)(j + 1) * total;
        const int kc = j + 1;
        const bool fused = kc <= KRYLOV_FUSED;
        if (mixed) {
            if (!have32) krylov_to_c64<<<cgrid, kBlock, 0, s>>>(total, qj, k->s32[0]);
            rc = he::apply_batched_gated(op, k->count, k->s32[0], k->s32[1], fields, velocity, HE_C64, gate, s);
            if (!fused) krylov_to_c128<<<cgrid, kBlock, 0, s>>>(total, k->s32[1], v);
        } else if (direction) {
            const double pair[6] = {fields[0], fields[1], fields[2], fields[0], fields[1], fields[2]};
            rc = he::apply_batched_gated(op, 2, qj, v, pair, 0, HE_C128, gate, s);
            if (!rc) rc = he::dipole_accumulate(op, qj + k->n / 2, v, direction, gate, s);
        } else {
            rc = he::apply_batched_gated(op, k->count, qj, v, fields, velocity, HE_C128, gate, s);
        }
        if (rc) break;
        have32 = false;
        if (fused) {   // three sweeps, the check in the second one's last block
            rc = fused_sweeps(k, kc, v, mixed ? k->s32[1] : nullptr, j, maxdim, dt, tol, s);
            if (rc) break;
            if (j + 1 < maxdim) {
                arnoldi_next_kernel<<<sweep_grid(k, reinterpret_cast<const void *>(arnoldi_next_kernel)), kBlock, 0, s>>>(
                    k->Q, k->n, k->qs(), kc, k->z, ld, v,
                                                               mixed ? k->s32[0] : nullptr, k->status);
                have32 = mixed;
            }
            HE_CUDA_TRY(cudaGetLastError());
            continue;
        }
        rc = krylov_cgs2(k, kc, v, k->H + (size_t)j * ld, k->H + (size_t)j * ld + j + 1, s, 1e-13);
        if (rc) break;
        arnoldi_check_kernel<<<k->count, 512, 0, s>>>(k->H, ld, k->hs(), j, maxdim, dt, tol, k->coef, k->work, k->ws(),
                                                      k->status);
        if (j + 1 < maxdim) normalize_kernel<<<bgrid(k), kBlock, 0, s>>>(v, v, k->n, k->status);
    }
    if (rc) return rc;
    // y = Q c with m from the status word; y is left as is when the solve failed
    combine_kernel<<<bgrid(k), kBlock, 0, s>>>(k->Q, k->n, k->qs(), k->coef, ld, static_cast<double2 *>(y), k->status, -1, 0);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

int expv_impl(he_krylov *k, he_handle op, const void *x, void *y, const double *fields, int velocity, double dt,
              double tol, int maxdim, int *dimension, double *estimate, int *converged, void *stream, int precision,
              const double *direction = nullptr)
{
    if (!k || !op || !x || !y || !fields) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    const size_t total = k->qs();   // one basis vector of every instance
    if (precision == HE_C64 && !k->s32[0]) {
        for (int q = 0; q < 2; ++q) HE_CUDA_TRY(cudaMalloc(&k->s32[q], total * sizeof(float2)));
    }
    if (maxdim < 1 || maxdim > k->maxdim) return he_fail(HE_ERR_ARG, "maxdim exceeds the workspace", __FILE__, __LINE__);
    if ((size_t)op->n * op->n * op->nc * (direction ? 2 : 1) != k->n)
        return he_fail(HE_ERR_SHAPE, "workspace size != operator size", __FILE__, __LINE__);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    // With graphs on, a solve whose configuration (operator, precision, gauge, maxdim) repeats
    // the previous one is captured on the workspace's own stream and replayed on the caller's
    // stream as one graph (the previous, uncaptured solve compiled and allocated everything
    // it needs); changed pointers and fields update the instantiated graph in place.
    const long long config = (long long)(reinterpret_cast<uintptr_t>(op) ^ ((uintptr_t)precision << 1) ^
                                         ((uintptr_t)velocity << 3) ^ ((uintptr_t)(direction != nullptr) << 4) ^
                                         ((uintptr_t)maxdim << 8));
    // Only the iterations a solve is likely to need are enqueued: two past the largest
    // dimension that solves of this configuration have converged at.  When the status read
    // after them shows a solve still running, the rest (up to maxdim) follow; the launches,
    // and so the results, are those of one solve enqueued to maxdim.
    if (k->hint_key != config) {
        k->hint_key = config;
        k->dim_seen = 0;
    }
    const int first = k->dim_seen > 0 ? std::min(maxdim, k->dim_seen + 2) : maxdim;
    const long long key = config ^ ((long long)first << 40);
    int rc;
    if (k->graphs && k->graph_key == key) {
        if (!k->capture_stream) HE_CUDA_TRY(cudaStreamCreateWithFlags(&k->capture_stream, cudaStreamNonBlocking));
        HE_CUDA_TRY(cudaStreamBeginCapture(k->capture_stream, cudaStreamCaptureModeRelaxed));
        rc = enqueue_expv(k, op, x, y, fields, velocity, dt, tol, maxdim, k->capture_stream, precision, direction, 0,
                          first);
        cudaGraph_t g = nullptr;
        const cudaError_t ended = cudaStreamEndCapture(k->capture_stream, &g);
        if (rc || ended != cudaSuccess || !g) {
            // The capture can be invalidated by work outside this solve (another host thread
            // loading its kernels, for instance): nothing captured has run, so drop it and
            // enqueue the solve directly.  A genuine error repeats there and is returned.
            // Captures that fail again and again (not a one-off invalidation) stop costing a
            // capture per solve: after KRYLOV_CAPTURE_RETRIES failures in a row the workspace
            // turns graphs off; he_krylov_capture_fallbacks reports the counts.
            if (g) cudaGraphDestroy(g);
            g = nullptr;
            cudaGetLastError();
            k->capture_fallbacks += 1;
            if (++k->capture_failures_in_row >= KRYLOV_CAPTURE_RETRIES) k->graphs = false;
            rc = enqueue_expv(k, op, x, y, fields, velocity, dt, tol, maxdim, s, precision, direction, 0, first);
        } else {
            k->capture_failures_in_row = 0;
            bool updated = false;
            if (k->graph_exec) {
                cudaGraphExecUpdateResultInfo info;
                updated = cudaGraphExecUpdate(k->graph_exec, g, &info) == cudaSuccess;
                if (!updated) {
                    cudaGetLastError();
                    cudaGraphExecDestroy(k->graph_exec);
                    k->graph_exec = nullptr;
                }
            }
            cudaError_t e = updated ? cudaSuccess : cudaGraphInstantiate(&k->graph_exec, g, 0);
            if (e == cudaSuccess) e = cudaGraphLaunch(k->graph_exec, s);
            if (e != cudaSuccess) rc = he_fail(HE_ERR_CUDA, cudaGetErrorString(e), __FILE__, __LINE__);
        }
        if (g) cudaGraphDestroy(g);
    } else {
        rc = enqueue_expv(k, op, x, y, fields, velocity, dt, tol, maxdim, s, precision, direction, 0, first);
    }
    if (rc) return rc;
    k->graph_key = key;
    if ((rc = krylov_read_status(k, s))) return rc;
    bool pending = false;
    for (int b = 0; b < k->count; ++b) pending = pending || !k->host_status[b].done;
    if (pending && first < maxdim) {
        rc = enqueue_expv(k, op, x, y, fields, velocity, dt, tol, maxdim, s, precision, direction, first, maxdim);
        if (rc) return rc;
        if ((rc = krylov_read_status(k, s))) return rc;
    }
    bool all = true;
    for (int b = 0; b < k->count; ++b) {
        const KrylovStatus &h = k->host_status[b];
        const bool ok = !h.failed && h.converged;
        if (ok) k->dim_seen = std::max(k->dim_seen, h.m);
        if (estimate) estimate[b] = h.estimate;
        if (dimension) dimension[b] = h.m;
        if (converged) converged[b] = ok;
        all = all && ok;
    }
    if (!all) return he_fail(HE_ERR_NOCONV, "Arnoldi did not converge", __FILE__, __LINE__);
    return HE_OK;
}
}  // namespace

namespace he {
// The first two sweeps of a fused CGS2 iteration for GMRES (no exponential check): H[:, j]
// gets the projections of v against Q_0..Q_{kc-1} and H[j+1, j] = h, v is updated once and
// the second projection stays in the workspace for krylov_next.  kc <= KRYLOV_FUSED.
int krylov_cgs2_fused(he_krylov *k, int kc, double2 *v, int j, cudaStream_t s, double happy_below)
{
    if (kc > KRYLOV_FUSED) return he_fail(HE_ERR_ARG, "fused CGS2 holds at most 16 vectors", __FILE__, __LINE__);
    return fused_sweeps(k, kc, v, nullptr, j, k->maxdim, 0.0, -1.0, s, happy_below);
}

// The third sweep: v <- (v - Q z') / h, the next basis vector (nothing once the solve is done).
int krylov_next(he_krylov *k, int kc, double2 *v, cudaStream_t s)
{
    arnoldi_next_kernel<<<sweep_grid(k, reinterpret_cast<const void *>(arnoldi_next_kernel)), kBlock, 0, s>>>(
        k->Q, k->n, k->qs(), kc, k->z, k->maxdim + 1, v, nullptr, k->status);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}
}  // namespace he

extern "C" int he_expv(he_krylov *k, he_handle op, const void *x, void *y, const double *field, int velocity,
                       double dt, double tol, int maxdim, int *dimension, double *estimate, void *stream)
{
    if (k && k->count != 1) return he_fail(HE_ERR_ARG, "batched workspace: use he_expv_batched", __FILE__, __LINE__);
    return expv_impl(k, op, x, y, field, velocity, dt, tol, maxdim, dimension, estimate, nullptr, stream, HE_C128);
}

extern "C" int he_expv_mixed(he_krylov *k, he_handle op, const void *x, void *y, const double *field, int velocity,
                             double dt, double tol, int maxdim, int *dimension, double *estimate, void *stream)
{
    if (k && k->count != 1) return he_fail(HE_ERR_ARG, "batched workspace: use he_expv_batched", __FILE__, __LINE__);
    return expv_impl(k, op, x, y, field, velocity, dt, tol, maxdim, dimension, estimate, nullptr, stream, HE_C64);
}

extern "C" int he_expv_batched(he_krylov *k, he_handle op, const void *x, void *y, const double *fields, int velocity,
                               double dt, double tol, int maxdim, int precision, int *dimension, double *estimate,
                               int *converged, void *stream)
{
    if (precision != HE_C128 && precision != HE_C64)
        return he_fail(HE_ERR_ARG, "precision must be HE_C128 or HE_C64", __FILE__, __LINE__);
    return expv_impl(k, op, x, y, fields, velocity, dt, tol, maxdim, dimension, estimate, converged, stream, precision);
}

// exp(-i dt B) x for B = [[H(field), direction . d], [0, H(field)]] (length gauge) on x = [u; w]
// (2 N complex128 values, a workspace of that length): y = [e^{-i dt H} u + L w; e^{-i dt H} w],
// L the derivative of e^{-i dt H(field)} along `direction` (the Frechet derivative of the
// exponential in the direction -i dt direction . d).  The fused Arnoldi of he_expv on the block
// operator: each Krylov vector costs one two-instance apply and one dipole pass.
extern "C" int he_expv_field_derivative(he_krylov *k, he_handle op, const void *x, void *y, const double *field,
                                        const double *direction, double dt, double tol, int maxdim, int *dimension,
                                        double *estimate, void *stream)
{
    if (!direction) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (k && k->count != 1) return he_fail(HE_ERR_ARG, "the derivative takes a single-instance workspace", __FILE__, __LINE__);
    return expv_impl(k, op, x, y, field, 0, dt, tol, maxdim, dimension, estimate, nullptr, stream, HE_C128, direction);
}
