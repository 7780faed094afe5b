/*
 * helium_b200.h — C-ABI of the B200 (sm_100a) two-electron helium propagation engine.
 *
 * Plain C types only: integers, doubles, raw pointers and sizes.  Complex arrays are
 * interleaved (re, im) pairs — the memory layout of numpy complex128 / C99 double
 * complex / torch.complex128 (and of complex64 when `precision` = HE_C64).  Wave
 * functions use the reference's Fortran order psi(i, j, c): r1 index fastest, then r2,
 * then channel (src/kernels.f90:125, python/native.py:25).  Device pointers and
 * `stream` (a cudaStream_t passed as void*) belong to the caller.  Every he_* entry
 * returns an int status (HE_OK = 0); he_last_error() gives the message of the last
 * failure on the calling thread.  Nothing here traps: device-side failures (e.g. a
 * Krylov or GMRES non-convergence) come back as status words.
 */
#ifndef HELIUM_B200_H
#define HELIUM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
    HE_OK = 0,
    HE_ERR_ARG = 1,        /* bad argument (null pointer, negative size, bad enum)        */
    HE_ERR_SHAPE = 2,      /* table inconsistent with its sizes (index out of range ...)  */
    HE_ERR_CUDA = 3,       /* CUDA runtime error; see he_last_error()                     */
    HE_ERR_NOCONV = 4,     /* Arnoldi or GMRES did not converge within its limits         */
    HE_ERR_UNSUPPORTED = 5,/* requested combination not built (e.g. no complex64 tables)  */
    HE_ERR_DEVICE = 6      /* a bounded device-side wait ran out (data not delivered)     */
};

enum { HE_C128 = 0, HE_C64 = 1 };   /* arithmetic of an apply: complex128 or complex64 */

/* ------------------------------------------------------------------------------------
 * Drop-in native symbol.
 * Replaces `tensor_apply` of the reference's Fortran library: src/kernels.f90:119-127
 * (bind(C) signature), loaded by python/native.py:8 and called at python/native.py:31-38
 * (callers python/helium3d.py:79-80, python/ground_s.py:46).  Same argument order and
 * meaning: scalars by value, zero-based CSR/edge indices, host column-major arrays,
 * `out` preallocated by the caller.  The work runs on the current CUDA device: the
 * tables and psi are staged to device memory, H·psi is computed in complex128 by the
 * sm_100a kernel and copied back.  The reference has no error channel; here a failure
 * leaves `out` untouched and is reported by he_last_status()/he_last_error().
 * ---------------------------------------------------------------------------------- */
void tensor_apply(int n, int nc, int nt, const int *ptr, const int *col, const double *tv,
                  const double *diag, int nv, const int *vptr, const int *vc, const int *vl,
                  const double *vcoef, const double *rad, int nd, const int *dptr, const int *dc,
                  const int *de, const double *dcoef, const double *ldiff, const double *r,
                  const double *field, int velocity, const double *psi, double *out);

int he_last_status(void);
const char *he_last_error(void);
int he_version(void);
/* binaryVersion of this library's kernels as loaded on the current device (100 = sm_100a);
 * a diagnostic of the build, no counterpart in the reference. */
int he_binary_version(int *version);

/* ------------------------------------------------------------------------------------
 * Device operator handle.
 * Replaces the construction half of the reference's TorchHamiltonian
 * (python/torch_backend.py:12-75): host tables in, device-resident tables out.
 * Tables are the arrays of python/helium3d.py:12-50 (or of CoupledHelium,
 * python/coupled_angular.py:13-55): kinetic CSR (ptr, col, tv), diagonal `diag`
 * (n*n*nc; may be NULL when the separable parts d1(n,nc), d2(n,nc) with
 * diag(i,j,c) = d1(i,c) + d2(j,c) are given), Coulomb edges (vptr, vc, vl, vcoef),
 * multipole radial table rad(n, n, nlam), dipole edges (dptr, dc, de, dcoef(3,nd),
 * ldiff) and nodes r(n).  flags: bit 0 = also build complex64 tables.
 * ---------------------------------------------------------------------------------- */
typedef struct he_operator *he_handle;

int he_create(he_handle *out, int n, int nc, int nt, const int *ptr, const int *col, const double *tv,
              const double *diag, const double *d1, const double *d2,
              int nv, const int *vptr, const int *vc, const int *vl, const double *vcoef,
              const double *rad, int nlam,
              int nd, const int *dptr, const int *dc, const int *de, const double *dcoef,
              const double *ldiff, const double *r, int flags);
int he_destroy(he_handle h);
int he_info(he_handle h, long long *values, int count);

/* out = H(field, gauge) psi.  Replaces TorchHamiltonian.apply
 * (python/torch_backend.py:109-131) and, bit for bit in meaning, kernels.f90:119-176.
 * velocity = 0: length gauge (field = E), 1: velocity gauge (field = A, adds |A|^2). */
int he_apply(he_handle h, const void *psi, void *out, const double *field, int velocity,
             int precision, void *stream);

/* out_b = H(fields[3b..3b+2], gauge) psi_b for count (<= 64) instances that share the
 * operator; psi and out hold the instances one after another (count x n*n*nc).  With the
 * banded and generated kernels available the whole batch is one launch per kernel, else
 * the instances run one at a time.  The reference applies one state at a time
 * (python/torch_backend.py:109-131); this batches its parameter-scan instances. */
int he_apply_batched(he_handle h, int count, const void *psi, void *out, const double *fields, int velocity,
                     int precision, void *stream);

/* out = psi + i*alpha*(H(field) psi - e_ref psi): the shifted Pade operator of
 * python/implicit.py:77-84 (K = H - E_ref, A(y) = y + i alpha K y), alpha complex. */
int he_apply_shifted(he_handle h, const void *psi, void *out, const double *field, int velocity,
                     double alpha_re, double alpha_im, double e_ref, int precision, void *stream);

/* Jacobi diagonal of H at zero field: diag + kinetic diagonals + same-channel Coulomb
 * (python/torch_backend.py:24-31).  out: n*n*nc complex128, device. */
int he_diagonal(he_handle h, void *out, void *stream);

/* ------------------------------------------------------------------------------------
 * tSURFF surface flux frame.  Replaces Helium.flux / TorchHamiltonian.flux
 * (python/helium3d.py:68-77, python/torch_backend.py:133-138):
 * frame(a, s, c) = sum_b J(s, lo+b) psi(a, lo+b, c)
 *   + sum_{electron-2 dipole edges k of c, |coef_k| > 1e-15} coef_k sum_b JP(s, lo+b) psi(a, lo+b, dc_k).
 * J, JP: ns x width complex128 row-major device arrays holding columns [lo, lo+width)
 * of surface_T and surface_P (python/helium3d.py:65-66); frame: (n, ns, nc) Fortran
 * order, complex128, device.
 * ---------------------------------------------------------------------------------- */
int he_flux(he_handle h, const void *psi, void *frame, int ns, int lo, int width, const void *J,
            const void *JP, const double *field, void *stream);

/* ------------------------------------------------------------------------------------
 * Krylov workspace and Arnoldi exponential.
 * Replaces exponential_action of python/propagate.py:6-39 and
 * python/torch_backend.py:140-158 (CGS2, H[j+1,j] = ||v||, happy breakdown below 1e-13,
 * checks at j >= 3 with (j+1) % 4 == 0 or j+1 == maxdim, c = expm(-i dt H_m)[:,0] beta,
 * err = |dt h_{m+1,m} c_m|).  The small exponential is evaluated on the device
 * (scaling and squaring, [13/13] Pade), so the host waits only at check points.
 * A workspace holds maxdim+1 basis vectors of n complex128 elements (plus maxdim
 * preconditioned directions when `flexible`), the Hessenberg matrix and scratch.
 * ---------------------------------------------------------------------------------- */
typedef struct he_krylov *he_krylov_handle;

int he_krylov_create(he_krylov_handle *out, long long n, int maxdim, int flexible);
int he_krylov_destroy(he_krylov_handle k);
/* Device address of basis vector j (which = 0: Q_j, which = 1: Z_j of flexible GMRES). */
int he_krylov_vector(he_krylov_handle k, int which, int j, void **ptr);

/* Arnoldi for an operator applied by the caller:
 *   he_krylov_start(x) -> beta (Q_0 = x / beta);
 *   for j: caller writes H Q_j into vector j+1, he_krylov_orthogonalize(j),
 *          he_expv_check(j, maxdim, dt, tol, sync) (normalises vector j+1 when not done);
 *   he_krylov_combine(m, y): y = Q[:, :m] c.
 * he_expv_check returns HE_ERR_NOCONV ("Arnoldi did not converge") when maxdim is
 * reached without meeting tol; with sync = 0 it does not block. */
int he_krylov_start(he_krylov_handle k, const void *x, double *beta, void *stream);
int he_krylov_orthogonalize(he_krylov_handle k, int j, void *stream);
int he_expv_check(he_krylov_handle k, int j, int maxdim, double dt, double tol, int sync, int *done, int *m,
                  double *estimate, void *stream);
int he_krylov_combine(he_krylov_handle k, int m, void *y, void *stream);

/* Fused y = exp(-i dt H(field)) x with the device operator `op` (no host work between
 * Krylov vectors).  x, y: n*n*nc complex128 device vectors, y != x.  All maxdim iterations
 * are enqueued; once the solve converges on the device, the remaining H·psi launches return
 * without work. */
int he_expv(he_krylov_handle k, he_handle op, const void *x, void *y, const double *field, int velocity,
            double dt, double tol, int maxdim, int *dimension, double *estimate, void *stream);
/* Mixed precision: as he_expv, but each H·psi runs in complex64 with FP32 accumulation
 * (the operator needs complex64 tables); the basis, CGS2, the Hessenberg exponential
 * and the error estimate stay complex128. */
int he_expv_mixed(he_krylov_handle k, he_handle op, const void *x, void *y, const double *field, int velocity,
                  double dt, double tol, int maxdim, int *dimension, double *estimate, void *stream);

/* Batched Arnoldi exponential: `count` (<= 64) instances that share the operator and the
 * time step, each with its own field (fields[3b..3b+2]), start vector and Krylov space,
 * advanced together (one launch per kernel per iteration for the whole batch).  The
 * workspace comes from he_krylov_create_batched (n = one instance's length); x and y hold
 * the instances one after another.  dimension/estimate/converged (optional, count
 * entries) report each instance; HE_ERR_NOCONV when any instance did not converge (its y
 * is untouched, the others are written).  precision as in he_apply.  The reference steps
 * one state at a time (python/propagate.py:6-50); this batches its parameter scans. */
int he_krylov_create_batched(he_krylov_handle *out, long long n, int maxdim, int count);
/* enable != 0: he_expv / he_expv_mixed / he_expv_batched / he_expv_field_derivative calls
 * that repeat the previous call's configuration (operator, precision, gauge, maxdim) are
 * captured once on an internal stream and replayed on the caller's stream as one CUDA graph, updated in place
 * for new states, fields and step sizes; results are identical.  Off by default. */
int he_krylov_set_graphs(he_krylov_handle k, int enable);
/* Solves whose graph capture was invalidated (by work outside the solve) and were enqueued
 * directly instead, and whether the workspace still captures: after three failed captures
 * in a row it stops trying.  No counterpart in the reference. */
int he_krylov_capture_fallbacks(he_krylov_handle k, int *fallbacks, int *graphs_on);
/* Field derivative of one step: y = exp(-i dt B) x for the block operator
 * B = [[H(field), direction . d], [0, H(field)]] (length gauge, complex128) on x = [u; w], so
 * y = [e^{-i dt H} u + L w; e^{-i dt H} w] with L the derivative of e^{-i dt H(field)} along
 * `direction` (d the dipole couplings).  The workspace holds vectors of 2 N.  Same fused
 * Arnoldi, checks and messages as he_expv.  Not part of the reference's interface: the
 * adjoint field gradient (one call per step of the backward sweep). */
int he_expv_field_derivative(he_krylov_handle k, he_handle op, const void *x, void *y, const double *field,
                             const double *direction, double dt, double tol, int maxdim, int *dimension,
                             double *estimate, void *stream);
int he_expv_batched(he_krylov_handle k, he_handle op, const void *x, void *y, const double *fields, int velocity,
                    double dt, double tol, int maxdim, int precision, int *dimension, double *estimate,
                    int *converged, void *stream);

/* FP64 throughput of the current device, for the compute roofline of H·psi: kind 0 = the
 * FP64 tensor pipe (mma.sync m8n8k4 f64, as in hpsi_band_kernel), kind 1 = FP64 FMA (as in
 * the mixing kernel).  Runs `iters` iterations of 8 independent chains on 4 CTAs per SM
 * and blocks until done.  Not part of the reference's interface. */
int he_fp64_peak(int kind, int iters, double *tflops, void *stream);

/* ------------------------------------------------------------------------------------
 * GMRES / CF4 building blocks (python/implicit.py:45-109).  The GMRES driver keeps its
 * Krylov basis in an he_krylov workspace (Q, and Z when flexible), orthogonalises with
 * he_krylov_orthogonalize, reads the Hessenberg column it needs for the small least
 * squares, and forms candidates and true residuals with these vector operations.
 * ---------------------------------------------------------------------------------- */
/* out = a x + b y (complex a, b); out may alias x or y. */
int he_vec_axpby(long long n, double a_re, double a_im, const void *x, double b_re, double b_im, const void *y,
                 void *out, void *stream);
/* *norm = ||b - t|| (t = NULL: ||b||); r = b - t is stored when r != NULL.  Blocks. */
int he_vec_residual_norm(long long n, const void *b, const void *t, void *r, double *norm, void *stream);
/* y = x / (1 + i alpha (diag + shift)): the Jacobi preconditioner of python/implicit.py:80,85. */
int he_vec_jacobi(long long n, const void *diag, double alpha_re, double alpha_im, double shift, const void *x,
                  void *y, void *stream);
/* Q_j (which = 0) or Z_j (which = 1) *= s. */
int he_krylov_scale(he_krylov_handle k, int which, int j, double s, void *stream);
/* Q_j /= h_{j,j-1} as left on the device by he_krylov_orthogonalize(j - 1) (no host read). */
int he_krylov_normalize(he_krylov_handle k, int j, void *stream);
/* Copy H[0:rows, j] (interleaved complex) to host memory `out`.  Blocks. */
int he_krylov_hessenberg(he_krylov_handle k, int j, int rows, void *out, void *stream);
/* H = 0 and a fresh status word (start of a GMRES cycle). */
int he_krylov_reset(he_krylov_handle k, void *stream);
/* y (+)= sum_{k<m} V_k c_k, V = Q (which = 0) or Z (which = 1), c: m host complex values. */
int he_krylov_combine_coef(he_krylov_handle k, int which, int m, const void *coef, void *y, int accumulate,
                           void *stream);

/* ------------------------------------------------------------------------------------
 * Mixed length/velocity gauge (replaces MixedHamiltonian, python/mixed_gauge.py:73-117).
 * he_set_mixed_gauge attaches, once per handle, the gauge-function profiles on the radial
 * grid (complex, n each: q = r (1 - f), qr2h = q / (2 r^2), F = r f, c0 = (1 - f)^2,
 * c2 = q'^2 - (1 - f)^2) and the quadratic angular edges per output channel (qptr: nc + 1,
 * source qc, electron qe (1 or 2), qcoef: 6 complex per edge = the projected
 * rhat_x^2, rhat_y^2, rhat_z^2, rhat_x rhat_y, rhat_x rhat_z, rhat_y rhat_z).
 * he_apply_mixed_terms adds to `out` (complex128, holding the field-free H psi) the
 * gauge terms of field = (A_x, A_y, A_z, E_x, E_y, E_z, then the six A_a A_b coefficients,
 * off-diagonal ones doubled), using the handle's dipole edges.
 * ---------------------------------------------------------------------------------- */
int he_set_mixed_gauge(he_handle h, const double *q, const double *qr2h, const double *F, const double *c0,
                       const double *c2, int nq, const int *qptr, const int *qc, const int *qe, const double *qcoef);
int he_apply_mixed_terms(he_handle h, const void *psi, void *out, const double *field, void *stream);
/* out += (direction . d) psi: the length-gauge dipole coupling of both electrons, i.e.
 * H(f + direction) psi - H(f) psi, complex128 (the field derivative of the Hamiltonian). */
int he_apply_dipole(he_handle h, const void *psi, void *out, const double *direction, void *stream);

/* ------------------------------------------------------------------------------------
 * He+ operator for the backward propagation of the tSURFF channel functions chi_c(t)
 * (replaces IonicAdjoint, python/ionic_adjoint.py:12-52, the device counterpart of the
 * sparse-LU SparseCF4 of python/implicit.py:111-123 used by python/streaming_surface.py:
 * 125-146).  H(c) = sum_k c_k M_k over nmat (<= 16) CSR planes sharing one pattern (ptr:
 * ndof+1, col: nnz, data: nmat x nnz interleaved complex), applied to nrhs (<= 16)
 * right-hand sides stored row-major x[row * nrhs + rhs].  he_ionic_apply: y = H(c) x, or
 * with shifted != 0 y = x + i alpha (H(c) x - shift x) (the shifted Pade operator).
 * he_ionic_set_preconditioner: na blocks of n rows (na n = ndof) with column-major n x n
 * eigenvectors S, inverses Si and eigenvalues E of each block of M_0;
 * he_ionic_precondition: y_a = S_a [(Si_a x_a) / (1 + i alpha (E_a + shift))].
 * ---------------------------------------------------------------------------------- */
typedef struct he_ionic *he_ionic_handle;
int he_ionic_create(he_ionic_handle *out, int ndof, int nrhs, int nmat, long long nnz, const int *ptr, const int *col,
                    const double *data);
int he_ionic_set_preconditioner(he_ionic_handle h, int na, int n, const double *S, const double *Si, const double *E);
int he_ionic_apply(he_ionic_handle h, const double *coef, int ncoef, const void *x, void *y, double alpha_re,
                   double alpha_im, double shift, int shifted, void *stream);
int he_ionic_precondition(he_ionic_handle h, const void *x, void *y, double alpha_re, double alpha_im, double shift,
                          void *stream);
int he_ionic_destroy(he_ionic_handle h);

/* ------------------------------------------------------------------------------------
 * Separable ionic resolvent preconditioner.  Replaces SeparablePreconditioner
 * (python/implicit.py:13-39): for channel c with one-electron momenta (l1[c], l2[c]),
 * Y_c = S_{l1} [ (S_{l1}^-1 Psi_c S_{l2}^-T) / (1 + i alpha (e_{l1}(i) + e_{l2}(j) + shift)) ] S_{l2}^T.
 * S, Sinv: nl column-major n x n complex128 matrices; evals: nl x n; the set-up
 * eigendecompositions are the caller's.  precision HE_C64 runs the products in
 * complex64 (the flexible-GMRES preconditioner of the reference) with complex128 in/out.
 * ---------------------------------------------------------------------------------- */
typedef struct he_separable *he_separable_handle;

int he_separable_create(he_separable_handle *out, int n, int nc, int nl, const double *S, const double *Sinv,
                        const double *evals, const int *l1, const int *l2, int precision);
int he_separable_destroy(he_separable_handle h);
int he_separable_apply(he_separable_handle h, const void *x, void *y, double alpha_re, double alpha_im,
                       double shift, void *stream);
/* Products per K slice of the complex64 preconditioner's TF32 tensor-core GEMMs: 3 (each
 * operand split into two TF32 parts, FP32-class accuracy; the default) or 1.  No
 * counterpart in the reference (its complex64 preconditioner runs cuBLAS/torch CGEMM). */
int he_separable_set_passes(he_separable_handle h, int passes);
/* Tile shape of the complex128 GEMMs (outputs per CTA): 0 = 64 x 128, 1 = 64 x 96,
 * 2 = 64 x 64, 3 = 32 x 64, 4 = 32 x 32, -1 = 64 x 64 when that grid fills two CTAs per
 * SM, else 32 x 32 (default); the project's autotuner
 * (SeparablePreconditioner.autotune) times them per operator.  No counterpart in the
 * reference. */
int he_separable_set_tile(he_separable_handle h, int shape);
/* HE_ERR_DEVICE once (then cleared) when a bounded pipeline wait of those GEMMs ran out. */
int he_separable_status(he_separable_handle h);

/* ------------------------------------------------------------------------------------
 * Device GMRES for one Pade system of CF4.  Replaces gmres (python/implicit.py:45-74) as
 * called by pade_step (:76-89): solves (I + i alpha (H(field) - e_ref)) x = b (velocity
 * gauge) from x0 = b, right preconditioned by `sep` (flexible GMRES when the workspace was
 * created flexible, for a complex64 `sep`) or, with sep NULL, by the Jacobi diagonal
 * 1 / (1 + i alpha (diag + shift)) of the device vector `diag`; restart length <= the
 * workspace's maxdim, at most max_restarts cycles; precision HE_C64 applies H in complex64
 * (inner solves of a mixed-precision solve; vectors stay complex128).  Least squares by
 * Givens rotations, the check points (every 4 iterations, flexible 2, and the restart
 * length), the true-residual acceptance and the restarts are decided on the device; the host
 * reads the state once per enqueued segment.  HE_ERR_NOCONV with the reference's message
 * 'GMRES did not converge: residual=..., iterations=...' when the cycles run out.
 * ---------------------------------------------------------------------------------- */
int he_gmres_shifted(he_krylov_handle k, he_handle op, he_separable_handle sep, const void *diag, const void *b,
                     void *x, const double *field, double alpha_re, double alpha_im, double e_ref, double shift,
                     double tol, int restart, int max_restarts, int precision, int *iterations, double *residual,
                     void *stream);

/* Diagnostic: in *iterations, the iterations the first segment of the next
 * he_gmres_shifted solve on k enqueues (the most a converged first cycle of the same
 * configuration needed; 0: the whole restart length) and, in *key when key != NULL, the
 * configuration it belongs to. */
int he_gmres_segment_hint(he_krylov_handle k, int *iterations, long long *key);

/* One CF4 step (python/implicit.py:91-109): y = the state x after dt, from the vector
 * potentials at the two Gauss points (fields: 2 x 3 host doubles, A(t + C1 dt) then
 * A(t + C2 dt), C1,2 = 1/2 -+ sqrt(3)/6).  Each of the two exponentials (field weights
 * (A2, A1) and (A1, A2), A1,2 = (3 -+ 2 sqrt 3)/12) is a [2/2] Pade pair of
 * he_gmres_shifted solves in complex128 with alpha = (dt/2)/(3 +- i sqrt 3), shift
 * a2 |A_eff|^2 - e_ref and the same preconditioner rule, followed by the phase
 * exp(-i dt (a2 (w . |A|^2 - |A_eff|^2 / 2) + e_ref / 2)).  x is not modified (x != y);
 * on HE_ERR_NOCONV ('GMRES did not converge') y is undefined and the caller halves dt as
 * python/implicit.py:104-109 does.  iterations: GMRES iterations of the four solves;
 * residual: the largest true relative residual.  The workspace k (as for he_gmres_shifted:
 * flexible for a complex64 preconditioner, restart <= its maxdim) also holds the step's
 * scratch vector, so concurrent steps need one workspace each. */
/* The host arithmetic of he_cf4_step (no device work): out[5 e .. 5 e + 4] for exponential
 * e = 0, 1 = the effective field (3), the preconditioner shift a2 |A_eff|^2 - e_ref and the
 * phase angle -dt (a2 (w . |A|^2 - |A_eff|^2 / 2) + e_ref / 2); out[10..13] = the two Pade
 * alphas (re, im).  out: 14 host doubles. */
int he_cf4_coefficients(const double *fields, double dt, double e_ref, double a2, double *out);
int he_cf4_step(he_krylov_handle k, he_handle op, he_separable_handle sep, const void *diag, const void *x, void *y,
                const double *fields, double dt, double e_ref, double a2, double tol, int restart, int max_restarts,
                int *iterations, double *residual, void *stream);

/* ------------------------------------------------------------------------------------
 * Online tSURFF (complex128).
 * he_surface_contract replaces SurfaceContractor.__call__ (python/surface_contract.py:41-56):
 *   q[j, o, s] = sum_{entries e of label j with eouter[e] = o} ecoef[e]
 *                sum_r conj(chi[(einner[e] n + r) nunique + column[j]]) frame[r fr + s fs + ecol[e] fc]
 * (entry lists per label, eptr[nlab+1], built from the reference's contraction set-up;
 * chi: (na n) x nunique row-major; frame strides in elements; q: (nlab, nouter, ns)
 * row-major).  he_volkov_add replaces VolkovAccumulator.add
 * (python/streaming_surface.py:54-64): current = i sqrt(2) (radial @ harmonics) phase,
 * radial[j,e,l] = sum_s q[j,l,s] tests[l,e,s], phase = exp(i (E_e t + k_e u_a.int_a + int_a2/2)),
 * amplitude += d (previous + current) / 2 unless `first`, previous = current.
 * All arrays are device arrays except int_a (3 host doubles).
 * ---------------------------------------------------------------------------------- */
int he_surface_contract(long long n, int nunique, int nlab, int nouter, int ns, const void *chi, const void *frame,
                        long long fr, long long fs, long long fc, const int *eptr, const int *ecol,
                        const int *einner, const double *ecoef, const int *eouter, const int *column, void *q,
                        void *stream);
int he_volkov_add(int nlab, int nouter, int ns, int ne, int nang, const void *q, const void *tests,
                  const void *harmonics, const double *energy, const double *k, const double *unit, double time,
                  const double *int_a, double int_a2, double d, int first, void *amplitude, void *previous,
                  void *stream);

/* ------------------------------------------------------------------------------------
 * One surface sample in one launch.  Replaces the per-sample chain of
 * python/streaming_surface.py:252-255 (flux frame python/helium3d.py:52-77 ->
 * SurfaceContractor.__call__ python/surface_contract.py:41-56 -> VolkovAccumulator.add
 * python/streaming_surface.py:54-64) with one cooperative launch: the frame of he_flux
 * (same arithmetic, written to `frame` as (c, s, r)), q of he_surface_contract (partial
 * sums per CTA, added in CTA order: reproducible, equal to he_surface_contract's q up to
 * summation order) written to `q`, and the Volkov update of he_volkov_add.
 * he_sample_create keeps the given device tables (stencil window J/JP, the contraction
 * entry lists, the Volkov tests/harmonics/energy/k/unit; the caller keeps them alive) and
 * allocates the per-CTA partial sums; ns <= 16 surface rows and nlab*nouter*ns <= 1024
 * (else HE_ERR_SHAPE).  The CTAs wait for each other's partial sums with a bounded poll:
 * when it runs out the sample is incomplete and he_sample_status reports HE_ERR_DEVICE
 * (once).  he_sample_grid: CTAs per launch.  The operator and the tables must outlive the
 * handle; the handle's partial sums serve one he_sample_record at a time (records on
 * several streams need one handle each).
 * ---------------------------------------------------------------------------------- */
typedef struct he_sample *he_sample_handle;
int he_sample_create(he_sample_handle *out, he_handle op, int ns, int lo, int width, const void *J, const void *JP,
                     int nunique, int nlab, int nouter, const int *eptr, const int *ecol, const int *einner,
                     const double *ecoef, const int *eouter, const int *column, int ne, int nang, const void *tests,
                     const void *harmonics, const double *energy, const double *k, const double *unit);
int he_sample_record(he_sample_handle h, const void *psi, const void *chi, const double *field, double time,
                     const double *int_a, double int_a2, double d, int first, void *frame, void *q, void *amplitude,
                     void *previous, void *stream);
int he_sample_grid(he_sample_handle h);
/* Test hook: later records wait for `extra` CTA arrivals that never come, so the bounded
 * wait runs out (about a second) and he_sample_status reports HE_ERR_DEVICE; 0 restores. */
int he_sample_set_wait_extra(he_sample_handle h, unsigned extra);
int he_sample_status(he_sample_handle h);
int he_sample_destroy(he_sample_handle h);

/* ------------------------------------------------------------------------------------
 * Run diagnostics on the device.  Replaces the checkpoint diagnostics of
 * python/run3d.py:212-224 (which copy the whole state to the host): out[0] = real-region
 * norm sum |u(i,j,c)|^2 f_i f_j with f = interior weight / |weight|, out[1] + i out[2] =
 * <g|psi> (0 when g is NULL), out[3] = exchange error ||u - P12 u|| with
 * (P12 u)(i,j,c) = sign_c u(j,i,xc_c) (python/coupled_angular.py:80-82).  f (n doubles),
 * xc (nc ints), sign (nc doubles) and the states are device memory; out is host memory.
 * ---------------------------------------------------------------------------------- */
int he_diagnostics(he_handle h, const void *psi, const void *g, const double *f, const int *xc, const double *sign,
                   double *out, void *stream);

/* ------------------------------------------------------------------------------------
 * Batched norms with no device allocation.  No counterpart in the reference: it serves
 * callers that cannot let a call allocate device memory (a process whose device memory
 * belongs to a pool allocator, a latency-critical loop that must not stall on the
 * allocator, a host runtime that forbids allocations outside its own allocator).
 * norms[v] = ||x + v*ld|| for v < count, count <= 64 (larger counts are rejected with
 * HE_ERR_ARG); x: complex128 device vectors of n elements; norms: host memory.  The
 * scratch is a fixed file-scope device array of 152,064 bytes, shared by all calls: calls
 * that overlap on the GPU race.  Under CUDA's default lazy module loading the driver
 * allocates that array on a device when the library first looks up its address there:
 * in he_create for the operator's device, else at the first he_vec_norms_noalloc call on
 * the device.  Make one of those before a pool allocator takes the device's memory and
 * before any stream capture on it (CUDA_MODULE_LOADING=EAGER allocates the array when
 * the context is created).  After that no call allocates device memory; the array stays
 * until the process exits.  Blocks the host until the norms are ready.
 * ---------------------------------------------------------------------------------- */
int he_vec_norms_noalloc(long long n, int count, const void *x, long long ld, double *norms, void *stream);

/* ------------------------------------------------------------------------------------
 * Operator set-up options and planner inspection (host only, no device work).
 * he_set_path: 1 = tiled kernels (default when the tables admit them; the kinetic part
 *   runs on the banded FP64 tensor-core kernel, TMA-staged, when psi is 16-byte aligned),
 *   3 = tiled kernels with the TMA-staged FMA kinetic kernel, 2 = tiled kernels with the
 *   shared-memory radial kernel (no TMA), 0 = generic gather kernel.
 * he_device_status: waits for the handle's device work and reports HE_ERR_DEVICE once
 *   (then clears it) when a bounded device-side wait of a kernel ran out.
 * he_plan_build / he_plan_array / he_plan_free expose the tiled plan of a set of tables.
 * ---------------------------------------------------------------------------------- */
int he_set_path(he_handle h, int tiled);
int he_device_status(he_handle h);
/* Length-gauge form of the banded kinetic kernel for one precision: stages 1 keeps one TMA
 * stage with the register budget of two CTAs per SM, 2 keeps two stages (the next box loads
 * during the current one).  Defaults: 1 for HE_C128, 2 for HE_C64 (the faster on B200).
 * Results are identical; the autotuner (B200Hamiltonian.autotune) times both.  No
 * counterpart in the reference. */
int he_set_band_stages(he_handle h, int precision, int stages);

/* ------------------------------------------------------------------------------------
 * Channel mixing: he_set_mix(h, 1) (default) uses the kernel generated for the handle's
 * coupling structure (every Coulomb and dipole edge unrolled, NVRTC-compiled for sm_100a
 * on the first tiled apply and cached by source); 0 uses the table-driven kernel.
 * he_mix_status: 0 not compiled yet, 1 generated kernel in use, -1 it failed to compile
 * (the table-driven kernel runs instead; he_last_error has the log).
 * he_set_mix_blocks(h, precision, b): size the generated kernel's register budget for b
 *   CTAs of 128 threads per SM (1..8; defaults 2 for HE_C128, 4 for HE_C64); the kernel is
 *   recompiled (or taken from the cache) on the next apply.  The autotuner of
 *   laqphysics_b200.engine (B200Hamiltonian.autotune) times the choices.
 * he_plan_mix_source / he_plan_mix_program / he_nvrtc_check: the generated source and the
 * mixing program (JSON) of a planner handle, and an NVRTC compile check for sm_100a
 * (host only).
 * ---------------------------------------------------------------------------------- */
int he_set_mix(he_handle h, int generated);
int he_mix_status(he_handle h);
int he_set_mix_blocks(he_handle h, int precision, int blocks);
long long he_plan_mix_source(void *plan, int dipole_real, char *buf, long long cap);
long long he_plan_mix_program(void *plan, char *buf, long long cap);
int he_nvrtc_check(const char *src, char *log, long long cap);
void *he_plan_build(int n, int nc, const int *ptr, const int *col, const double *tv, int nv, const int *vptr,
                    const int *vc, const int *vl, const double *vcoef, int nlam, int nd, const int *dptr,
                    const int *dc, const int *de, const double *r);
long long he_plan_array(void *plan, int which, void *dst);
void he_plan_free(void *plan);

#ifdef __cplusplus
}
#endif
#endif /* HELIUM_B200_H */
