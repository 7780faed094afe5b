// Two-electron H·psi on sm_100a.
//
// out(i,j,c) = beta*psi(i,j,c) + gamma*(H psi)(i,j,c) with
//   (H psi) = diag psi + T_1 psi + T_2 psi + sum_{Coulomb edges of c} vcoef rad_lam psi_c'
//           + dipole edges (length: coef r psi_s, velocity: i coef (ldiff/(2r) psi_s + [T, r] psi_s))
//           + |A|^2 psi (velocity gauge),
// i.e. the operator of the reference's src/kernels.f90:119-176 and
// python/torch_backend.py:109-131.  (beta, gamma) = (0, 1) is the plain apply;
// (1 - i*alpha*E_ref, i*alpha) is the shifted Pade operator of python/implicit.py:77-84.
#include "common.cuh"
#include "hamiltonian.cuh"

namespace he {

// ---------------------------------------------------------------------------------
// Gather kernel: one thread per output amplitude, lanes along r1 (coalesced).
// Generic over the tables (full or separable diagonal, any CSR / edge lists).
// ---------------------------------------------------------------------------------
template <typename R, bool SEP, bool VEL>
__global__ void __launch_bounds__(256)
hpsi_gather_kernel(DeviceTables<R> t, const cplx<R> *__restrict__ psi, cplx<R> *__restrict__ out,
                   R f0, R f1, R f2, cplx<R> beta, cplx<R> gamma)
{
    const int n = t.n;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int c = blockIdx.z;
    if (i >= n || j >= n) return;
    const size_t nn = (size_t)n * n;
    const size_t p = (size_t)i + (size_t)n * j;
    const cplx<R> *pc = psi + nn * c;
    const cplx<R> x = pc[p];
    const cplx<R> d = SEP ? cadd<R>(ldg<R>(t.d1 + i + (size_t)n * c), ldg<R>(t.d2 + j + (size_t)n * c))
                          : ldg<R>(t.diag + p + nn * c);
    cplx<R> val = cmul<R>(d, x);
    for (int k = __ldg(t.ptr + i), e = __ldg(t.ptr + i + 1); k < e; ++k)
        val = cfma<R>(ldg<R>(t.tv + k), pc[__ldg(t.col + k) + (size_t)n * j], val);
    for (int k = __ldg(t.ptr + j), e = __ldg(t.ptr + j + 1); k < e; ++k)
        val = cfma<R>(ldg<R>(t.tv + k), pc[i + (size_t)n * __ldg(t.col + k)], val);
    for (int k = __ldg(t.vptr + c), e = __ldg(t.vptr + c + 1); k < e; ++k) {
        const cplx<R> w = cmul<R>(ldg<R>(t.vcoef + k), ldg<R>(t.rad + p + nn * __ldg(t.vl + k)));
        val = cfma<R>(w, psi[p + nn * __ldg(t.vc + k)], val);
    }
    for (int k = __ldg(t.dptr + c), e = __ldg(t.dptr + c + 1); k < e; ++k) {
        const cplx<R> *dk = t.dcoef + 3 * (size_t)k;
        cplx<R> coef = cscale<R>(f0, ldg<R>(dk));
        coef = rfma<R>(f1, ldg<R>(dk + 1), coef);
        coef = rfma<R>(f2, ldg<R>(dk + 2), coef);
        if (sqrt(cabs2<R>(coef)) < (R)1e-30) continue;
        const int s = __ldg(t.dc + k);
        const cplx<R> *ps = psi + nn * s;
        const bool first = __ldg(t.de + k) == 1;
        const int a = first ? i : j;           // coordinate the dipole acts on
        const cplx<R> ra = ldg<R>(t.r + a);
        if (!VEL) {
            val = cfma<R>(cmul<R>(coef, ra), ps[p], val);
        } else {
            cplx<R> part = mk<R>(0, 0);
            const R ld = __ldg(t.ldiff + k);
            if (ld != (R)0)   // ldiff / (2 r_a) psi_s, with 1/(2 r) tabulated on the host
                part = cmul<R>(cscale<R>(ld, ldg<R>(t.hinv + a)), ps[p]);
            for (int q = __ldg(t.ptr + a), e2 = __ldg(t.ptr + a + 1); q < e2; ++q) {
                const int b = __ldg(t.col + q);
                const cplx<R> w = cmul<R>(ldg<R>(t.tv + q), csub<R>(ldg<R>(t.r + b), ra));
                const cplx<R> src = first ? ps[b + (size_t)n * j] : ps[i + (size_t)n * b];
                part = cfma<R>(w, src, part);
            }
            // i * coef * part
            val = cfma<R>(mk<R>(-coef.y, coef.x), part, val);
        }
    }
    if (VEL) {
        const R a2 = f0 * f0 + f1 * f1 + f2 * f2;
        val = rfma<R>(a2, x, val);
    }
    out[p + nn * c] = cfma<R>(gamma, val, cmul<R>(beta, x));
}

template <typename R>
int launch_hpsi(const DeviceTables<R> &t, const cplx<R> *psi, cplx<R> *out, const double *field, int velocity,
                cplx<R> beta, cplx<R> gamma, cudaStream_t stream)
{
    const dim3 block(32, 8);
    const dim3 grid((t.n + 31) / 32, (t.n + 7) / 8, t.nc);
    const R f0 = (R)field[0], f1 = (R)field[1], f2 = (R)field[2];
    if (t.diag_separable) {
        if (velocity) hpsi_gather_kernel<R, true, true><<<grid, block, 0, stream>>>(t, psi, out, f0, f1, f2, beta, gamma);
        else hpsi_gather_kernel<R, true, false><<<grid, block, 0, stream>>>(t, psi, out, f0, f1, f2, beta, gamma);
    } else {
        if (velocity) hpsi_gather_kernel<R, false, true><<<grid, block, 0, stream>>>(t, psi, out, f0, f1, f2, beta, gamma);
        else hpsi_gather_kernel<R, false, false><<<grid, block, 0, stream>>>(t, psi, out, f0, f1, f2, beta, gamma);
    }
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

template int launch_hpsi<double>(const DeviceTables<double> &, const double2 *, double2 *, const double *, int,
                                 double2, double2, cudaStream_t);
template int launch_hpsi<float>(const DeviceTables<float> &, const float2 *, float2 *, const double *, int,
                                float2, float2, cudaStream_t);

// ---------------------------------------------------------------------------------
// Jacobi diagonal (python/torch_backend.py:24-31): diag + T_ii + T_jj + same-channel
// Coulomb multipoles, evaluated at zero field.
// ---------------------------------------------------------------------------------
__global__ void diagonal_kernel(DeviceTables<double> t, const double2 *__restrict__ tdiag, double2 *__restrict__ out)
{
    const int n = t.n;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int c = blockIdx.z;
    if (i >= n || j >= n) return;
    const size_t nn = (size_t)n * n;
    const size_t p = (size_t)i + (size_t)n * j;
    double2 d = t.diag_separable ? cadd<double>(t.d1[i + (size_t)n * c], t.d2[j + (size_t)n * c]) : t.diag[p + nn * c];
    d = cadd<double>(d, cadd<double>(tdiag[i], tdiag[j]));
    for (int k = t.vptr[c]; k < t.vptr[c + 1]; ++k)
        if (t.vc[k] == c) d = cadd<double>(d, cmul<double>(t.vcoef[k], t.rad[p + nn * t.vl[k]]));
    out[p + nn * c] = d;
}

int launch_diagonal(const DeviceTables<double> &t, const double2 *tdiag, double2 *out, cudaStream_t stream)
{
    const dim3 block(32, 8);
    const dim3 grid((t.n + 31) / 32, (t.n + 7) / 8, t.nc);
    diagonal_kernel<<<grid, block, 0, stream>>>(t, tdiag, out);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

}  // namespace he
