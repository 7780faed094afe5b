/*
 * ORACLE — test infrastructure only.  Nothing in the product path links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg (and its `--impl reference` arm) use the library built from it, as the checker
 * and as the timed CPU baseline.
 *
 * Plain C99 + OpenMP restatement of the reference's native two-electron H·psi,
 * `tensor_apply` in src/kernels.f90:119-176 (bind(C) symbol loaded by
 * python/native.py:8 and called from python/native.py:24-38).  The Fortran source
 * cannot be compiled here (no Fortran front end), so this restatement is the CPU
 * oracle and the `cpu_baseline` "port".  It keeps:
 *   - the exact C signature and argument order of kernels.f90:119-127
 *     (scalars by value, zero-based indices, column-major arrays);
 *   - the per-output accumulation order of kernels.f90:132-171, term by term;
 *   - the `abs(coef) < 1e-30` skip of kernels.f90:145 and the `ldiff /= 0`
 *     branches of kernels.f90:156 and :162;
 *   - Fortran complex arithmetic (built with -fcx-fortran-rules, no NaN recovery).
 * Parity of this file is pinned by tests/test_oracle.py against the reference's
 * independent Kronecker assembly (python/helium3d.py:105-123) stored as golden
 * fixtures under tests/golden/ by tests/golden/make_golden.py.
 */
#include <complex.h>
#include <math.h>
#include <stddef.h>

typedef double complex zd;

/* psi(i,j,c) with i fastest: kernels.f90:125 declares psi(n,n,nc). */
#define IDX(i, j, c) ((size_t)(i) + (size_t)n * ((size_t)(j) + (size_t)n * (size_t)(c)))

/* Output channels [c_begin, c_end) of H·psi; tensor_apply is the full range.  The
 * partial range lets the timed CPU baseline run a bounded sample of a large case. */
void tensor_apply_channels(int n, int nc, int nt, const int *ptr, const int *col, const zd *tv,
                           const zd *diag, int nv, const int *vptr, const int *vc, const int *vl,
                           const zd *vcoef, const zd *rad, int nd, const int *dptr, const int *dc,
                           const int *de, const zd *dcoef, const double *ldiff, const zd *r,
                           const double *field, int velocity, const zd *psi, zd *out,
                           int c_begin, int c_end)
{
    (void)nt; (void)nv; (void)nd; (void)nc;
    const double a2 = field[0] * field[0] + field[1] * field[1] + field[2] * field[2];
    /* kernels.f90:130 — OpenMP over (c, j) collapsed, i innermost. */
#pragma omp parallel for collapse(2) schedule(static)
    for (int c = c_begin; c < c_end; ++c) {
        for (int j = 0; j < n; ++j) {
            for (int i = 0; i < n; ++i) {
                zd val = diag[IDX(i, j, c)] * psi[IDX(i, j, c)];                 /* :134 */
                for (int k = ptr[i]; k < ptr[i + 1]; ++k)                        /* :135-137 */
                    val = val + tv[k] * psi[IDX(col[k], j, c)];
                for (int k = ptr[j]; k < ptr[j + 1]; ++k)                        /* :138-140 */
                    val = val + tv[k] * psi[IDX(i, col[k], c)];
                for (int k = vptr[c]; k < vptr[c + 1]; ++k)                      /* :141-143 */
                    val = val + vcoef[k] * rad[IDX(i, j, vl[k])] * psi[IDX(i, j, vc[k])];
                for (int k = dptr[c]; k < dptr[c + 1]; ++k) {                    /* :144-169 */
                    const zd coef = field[0] * dcoef[3 * (size_t)k] + field[1] * dcoef[3 * (size_t)k + 1]
                                  + field[2] * dcoef[3 * (size_t)k + 2];
                    if (cabs(coef) < 1e-30) continue;                            /* :145 */
                    const int s = dc[k];
                    if (velocity == 0) {
                        if (de[k] == 1) val = val + coef * r[i] * psi[IDX(i, j, s)];
                        else            val = val + coef * r[j] * psi[IDX(i, j, s)];
                    } else {
                        zd part = 0;
                        if (de[k] == 1) {
                            if (ldiff[k] != 0) part = ldiff[k] / (2 * r[i]) * psi[IDX(i, j, s)];
                            for (int a = ptr[i]; a < ptr[i + 1]; ++a)
                                part = part + tv[a] * (r[col[a]] - r[i]) * psi[IDX(col[a], j, s)];
                        } else {
                            if (ldiff[k] != 0) part = ldiff[k] / (2 * r[j]) * psi[IDX(i, j, s)];
                            for (int a = ptr[j]; a < ptr[j + 1]; ++a)
                                part = part + tv[a] * (r[col[a]] - r[j]) * psi[IDX(i, col[a], s)];
                        }
                        val = val + I * coef * part;                              /* :168 */
                    }
                }
                if (velocity == 1) val = val + a2 * psi[IDX(i, j, c)];           /* :170 */
                out[IDX(i, j, c)] = val;
            }
        }
    }
}

void tensor_apply(int n, int nc, int nt, const int *ptr, const int *col, const zd *tv,
                  const zd *diag, int nv, const int *vptr, const int *vc, const int *vl,
                  const zd *vcoef, const zd *rad, int nd, const int *dptr, const int *dc,
                  const int *de, const zd *dcoef, const double *ldiff, const zd *r,
                  const double *field, int velocity, const zd *psi, zd *out)
{
    tensor_apply_channels(n, nc, nt, ptr, col, tv, diag, nv, vptr, vc, vl, vcoef, rad, nd, dptr, dc, de,
                          dcoef, ldiff, r, field, velocity, psi, out, 0, nc);
}

/* Thread count the OpenMP runtime will use; reported beside CPU-baseline timings. */
int oracle_max_threads(void)
{
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}
