// Mixed length/velocity gauge terms (the reference's MixedHamiltonian, python/mixed_gauge.py:
// 73-117).  With the gauge function f(r) (1 inside, 0 beyond the switch) and q = r (1 - f),
// the operator is the field-free Hamiltonian plus, per electron e (coordinate r_e),
//   i (A.d_k) [ (Bq psi_s)(r_e) + ldiff_k q/(2 r^2)(r_e) psi_s ] + (E.d_k) r f(r_e) psi_s
//   + 1/2 (Q.S_k) c2(r_e) psi_s + 1/2 (A.A) c0(r_e) psi
// over the dipole edges k (d_k the Cartesian coefficients) and the quadratic edges k (S_k the
// six projected rhat_a rhat_b, Q the coefficients A_a A_b), Bq = [T, q], c0 = (1 - f)^2,
// c2 = q'^2 - (1 - f)^2.  This kernel adds those terms to an output that already holds the
// field-free H psi (one thread per point and output channel).
#include "common.cuh"
#include "operator.cuh"

namespace {

struct MixedField {
    double A[3], E[3], Q[6];
};

__global__ void mixed_gauge_kernel(he::DeviceTables<double> t, const double2 *__restrict__ q,
                                   const double2 *__restrict__ qr2h, const double2 *__restrict__ F,
                                   const double2 *__restrict__ c0, const double2 *__restrict__ c2,
                                   const int *__restrict__ qptr, const int *__restrict__ qc, const int *__restrict__ qe,
                                   const double2 *__restrict__ qcoef, MixedField f, const double2 *__restrict__ psi,
                                   double2 *__restrict__ out)
{
    const int n = t.n;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int c = blockIdx.z;
    if (i >= n || j >= n) return;
    const size_t nn = (size_t)n * n;
    const size_t p = (size_t)i + (size_t)n * j;
    double2 val = mk<double>(0, 0);
    for (int k = t.dptr[c]; k < t.dptr[c + 1]; ++k) {
        const double2 *dk = t.dcoef + 3 * (size_t)k;
        double2 cA = mk<double>(0, 0), cE = mk<double>(0, 0);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            cA = rfma<double>(f.A[a], dk[a], cA);
            cE = rfma<double>(f.E[a], dk[a], cE);
        }
        const double2 *ps = psi + nn * t.dc[k];
        const bool first = t.de[k] == 1;
        const int a = first ? i : j;
        const double2 qa = q[a];
        double2 part = cscale<double>(t.ldiff[k], cmul<double>(qr2h[a], ps[p]));
        for (int e = t.ptr[a]; e < t.ptr[a + 1]; ++e) {
            const int b = t.col[e];
            const double2 w = cmul<double>(t.tv[e], csub<double>(q[b], qa));
            part = cfma<double>(w, first ? ps[b + (size_t)n * j] : ps[i + (size_t)n * b], part);
        }
        val = cfma<double>(mk<double>(-cA.y, cA.x), part, val);          // i (A.d) part
        val = cfma<double>(cmul<double>(cE, F[a]), ps[p], val);         // (E.d) r f psi_s
    }
    for (int k = qptr[c]; k < qptr[c + 1]; ++k) {
        const double2 *sk = qcoef + 6 * (size_t)k;
        double2 cQ = mk<double>(0, 0);
#pragma unroll
        for (int m = 0; m < 6; ++m) cQ = rfma<double>(f.Q[m], sk[m], cQ);
        const int a = qe[k] == 1 ? i : j;
        val = cfma<double>(cscale<double>(0.5, cmul<double>(cQ, c2[a])), psi[p + nn * qc[k]], val);
    }
    const double2 x = psi[p + nn * c];
    const double q2 = 0.5 * (f.Q[0] + f.Q[1] + f.Q[2]);
    val = cfma<double>(cscale<double>(q2, cadd<double>(c0[i], c0[j])), x, val);
    out[p + nn * c] = cadd<double>(out[p + nn * c], val);
}

// out(p, c) += sum over the dipole edges k of channel c of (direction . d_k) r(a) psi(p, src_k), a the
// coordinate of the edge's electron (i for electron 1, j for electron 2): the length-gauge field
// coupling of both electrons, i.e. H(f + direction) psi - H(f) psi.  One thread per point and
// output channel; returns at once while *skip != 0.
__global__ void dipole_kernel(he::DeviceTables<double> t, double dx, double dy, double dz,
                              const double2 *__restrict__ psi, double2 *__restrict__ out, const int *skip)
{
    if (skip && *skip) return;
    const int n = t.n, c = blockIdx.y;
    const size_t nn = (size_t)n * n;
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nn || t.dptr[c] == t.dptr[c + 1]) return;
    const int i = (int)(p % n), j = (int)(p / n);
    double2 val = mk<double>(0, 0);
    for (int k = t.dptr[c]; k < t.dptr[c + 1]; ++k) {
        const double2 *dk = t.dcoef + 3 * (size_t)k;
        double2 coef = cscale<double>(dx, dk[0]);
        coef = rfma<double>(dy, dk[1], coef);
        coef = rfma<double>(dz, dk[2], coef);
        val = cfma<double>(cmul<double>(coef, t.r[t.de[k] == 1 ? i : j]), psi[p + nn * t.dc[k]], val);
    }
    out[p + nn * c] = cadd<double>(out[p + nn * c], val);
}

template <typename T> int upload(he_operator *h, T **dst, const void *src, size_t count)
{
    *dst = nullptr;
    if (!count) return HE_OK;
    HE_CUDA_TRY(cudaMalloc(dst, count * sizeof(T)));
    h->allocations.push_back(*dst);
    HE_CUDA_TRY(cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice));
    return HE_OK;
}

}  // namespace

extern "C" int he_set_mixed_gauge(he_handle h, const double *q, const double *qr2h, const double *F, const double *c0,
                                  const double *c2, int nq, const int *qptr, const int *qc, const int *qe,
                                  const double *qcoef)
{
    if (!h || !q || !qr2h || !F || !c0 || !c2 || !qptr || nq < 0 || (nq > 0 && (!qc || !qe || !qcoef)))
        return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (qptr[0] != 0 || qptr[h->nc] != nq) return he_fail(HE_ERR_SHAPE, "quadratic edge pointer does not span nq", __FILE__, __LINE__);
    for (int k = 0; k < nq; ++k)
        if (qc[k] < 0 || qc[k] >= h->nc || (qe[k] != 1 && qe[k] != 2))
            return he_fail(HE_ERR_SHAPE, "quadratic edge out of range", __FILE__, __LINE__);
    int rc;
    const size_t n = h->n;
    if ((rc = upload<double2>(h, &h->mg.q, q, n)) || (rc = upload<double2>(h, &h->mg.qr2h, qr2h, n)) ||
        (rc = upload<double2>(h, &h->mg.F, F, n)) || (rc = upload<double2>(h, &h->mg.c0, c0, n)) ||
        (rc = upload<double2>(h, &h->mg.c2, c2, n)) || (rc = upload<int>(h, &h->mg.qptr, qptr, h->nc + 1)) ||
        (rc = upload<int>(h, &h->mg.qc, qc, nq)) || (rc = upload<int>(h, &h->mg.qe, qe, nq)) ||
        (rc = upload<double2>(h, &h->mg.qcoef, qcoef, 6 * (size_t)nq)))
        return rc;
    h->mg.nq = nq;
    h->mg.ready = true;
    return HE_OK;
}

extern "C" int he_apply_mixed_terms(he_handle h, const void *psi, void *out, const double *field, void *stream)
{
    if (!h || !psi || !out || !field) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (!h->mg.ready) return he_fail(HE_ERR_ARG, "mixed gauge tables not set (he_set_mixed_gauge)", __FILE__, __LINE__);
    MixedField f;
    for (int a = 0; a < 3; ++a) { f.A[a] = field[a]; f.E[a] = field[3 + a]; }
    for (int m = 0; m < 6; ++m) f.Q[m] = field[6 + m];
    const dim3 block(32, 8);
    const dim3 grid((h->n + 31) / 32, (h->n + 7) / 8, h->nc);
    mixed_gauge_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        h->t64, h->mg.q, h->mg.qr2h, h->mg.F, h->mg.c0, h->mg.c2, h->mg.qptr, h->mg.qc, h->mg.qe, h->mg.qcoef, f,
        static_cast<const double2 *>(psi), static_cast<double2 *>(out));
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

namespace he {
int dipole_accumulate(he_operator *h, const double2 *psi, double2 *out, const double direction[3], const int *skip,
                      cudaStream_t stream)
{
    if (!h->t64.r || h->nd < 1) return he_fail(HE_ERR_UNSUPPORTED, "operator has no dipole couplings", __FILE__, __LINE__);
    const size_t nn = (size_t)h->n * h->n;
    const dim3 grid((unsigned)((nn + 255) / 256), h->nc);
    dipole_kernel<<<grid, 256, 0, stream>>>(h->t64, direction[0], direction[1], direction[2], psi, out, skip);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}
}  // namespace he

extern "C" int he_apply_dipole(he_handle h, const void *psi, void *out, const double *direction, void *stream)
{
    if (!h || !psi || !out || !direction) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (psi == out) return he_fail(HE_ERR_ARG, "the dipole coupling cannot run in place", __FILE__, __LINE__);
    return he::dipole_accumulate(h, static_cast<const double2 *>(psi), static_cast<double2 *>(out), direction, nullptr,
                                 static_cast<cudaStream_t>(stream));
}
