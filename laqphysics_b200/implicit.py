"""CF4 Magnus + [2/2] Pade time step with device GMRES (drop-in for python/implicit.py).

Same functions, signatures, constants, messages and acceptance rules as the
reference (python/implicit.py:13-109):

* ``SeparablePreconditioner(engine, precision)``: exact resolvent of the two uncoupled
  ionic radial Hamiltonians; the eigendecompositions are set-up work on the host
  (scipy, with the reference's 1e12 condition limit); each application is four
  batched n^3 GEMMs per channel plus a resolvent scaling on the device.
* ``gmres``: right-preconditioned GMRES (restart 32) or flexible GMRES (restart 16)
  when the preconditioner is complex64; CGS2 Arnoldi on the device; least squares
  every 4 (flexible: 2) iterations; a solution is accepted only on its TRUE residual.
* ``pade_step`` / ``cf4_step``: the two Pade roots 3 +- i sqrt(3), CF4 fields at the
  Gauss points, the scalar |A|^2 and E_ref phases, and dt halving (depth <= 6) on
  'GMRES did not converge'.
* ``precision='mixed'`` (pade_step / cf4_step): complex128 defect correction around
  complex64 inner GMRES solves (complex64 H·psi with FP32 accumulation); an addition, the
  reference has one precision.
The operator y + i alpha (H - E_ref) y is one fused launch of the engine.
"""
import ctypes as ct

import numpy as np
import torch
from scipy.linalg import eig, inv

from ._lib import LIB, HE_C128, HE_C64, HE_ERR_NOCONV, check
from .engine import _stream
from .torch_backend import workspace

SQRT3 = np.sqrt(3.)
C1 = .5 - SQRT3 / 6
C2 = .5 + SQRT3 / 6
A1 = (3 - 2 * SQRT3) / 12
A2 = (3 + 2 * SQRT3) / 12


def _vp(t):
    return ct.c_void_p(t.data_ptr())


def norm(x):
    value = ct.c_double()
    check(LIB.he_vec_residual_norm(x.numel(), _vp(x), None, None, ct.byref(value), _stream(x.device)), 'norm')
    return value.value


def axpby(a, x, b, y, out=None):
    """out = a x + b y (complex scalars) on the device."""
    out = torch.empty_like(x) if out is None else out
    a, b = complex(a), complex(b)
    check(LIB.he_vec_axpby(x.numel(), a.real, a.imag, _vp(x), b.real, b.imag, _vp(y), _vp(out), _stream(x.device)),
          'axpby')
    return out


class SeparablePreconditioner:
    """Exact resolvent of H1(l1) + H2(l2) (python/implicit.py:13-39)."""

    def __init__(self, engine, precision='complex128'):
        h = engine.h
        self.engine = engine
        labels = [tuple(b[:2]) for b in h.basis] if hasattr(h, 'basis') else [(a[0], b[0]) for a, b in h.ch]
        maxl = max(max(p) for p in labels)
        T = h.grid.kinetic.toarray()
        r = h.r
        values, vectors, inverses, conditions = [], [], [], []
        for l in range(maxl + 1):
            H = T + np.diag(-2 * h.cut / r + l * (l + 1) / (2 * r * r))
            e, S = eig(H)
            conditions.append(float(np.linalg.cond(S)))
            values.append(e); vectors.append(S); inverses.append(inv(S))
        if max(conditions) > 1e12:
            raise RuntimeError('ionic eigenbasis too ill-conditioned for separable preconditioner')
        if precision not in ('complex128', 'complex64'):
            raise ValueError('invalid preconditioner precision')
        self.condition_numbers = conditions
        self.precision = precision
        self.flexible = precision == 'complex64'
        self.dtype = torch.complex64 if self.flexible else torch.complex128
        col_major = lambda mats: np.ascontiguousarray(np.array([m.T for m in mats]), dtype=np.complex128)
        S, I = col_major(vectors), col_major(inverses)
        ev = np.ascontiguousarray(np.array(values), dtype=np.complex128)
        l1 = np.array([a for a, _ in labels], np.int32)
        l2 = np.array([b for _, b in labels], np.int32)
        handle = ct.c_void_p()
        with torch.cuda.device(engine.device):
            check(LIB.he_separable_create(ct.byref(handle), h.n, h.nc, maxl + 1, S.ctypes.data, I.ctypes.data,
                                          ev.ctypes.data, l1.ctypes.data, l2.ctypes.data,
                                          HE_C64 if self.flexible else HE_C128), 'he_separable_create')
        self.handle = handle

    def autotune(self, repeats=3):
        """Time the complex128 GEMM tile shapes (he_separable_set_tile 0..4) on this
        operator and keep the fastest; returns {shape: ms per apply}.  complex64 has one
        shape (128 x up to 256 tcgen05 tiles) and returns {}."""
        if self.flexible:
            return {}
        n = self.engine.h.size
        x = torch.randn(n, dtype=torch.complex128, device=self.engine.device)
        alpha = .05 / (3 + 1j * SQRT3)
        times = {}
        for shape in range(5):
            check(LIB.he_separable_set_tile(self.handle, shape), 'he_separable_set_tile')
            self.apply(x, alpha, -2.)
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            for _ in range(repeats):
                self.apply(x, alpha, -2.)
            stop.record()
            stop.synchronize()
            times[shape] = start.elapsed_time(stop) / repeats
        best = min(times, key=times.get)
        check(LIB.he_separable_set_tile(self.handle, best), 'he_separable_set_tile')
        self.tile_times, self.tile = times, best
        return times

    def apply(self, x, alpha, shift):
        y = torch.empty_like(x)
        alpha = complex(alpha)
        check(LIB.he_separable_apply(self.handle, _vp(x), _vp(y), alpha.real, alpha.imag, float(shift),
                                     _stream(x.device)), 'he_separable_apply')
        return y

    def __del__(self):
        handle = getattr(self, 'handle', None)
        if handle is not None and handle.value:
            LIB.he_separable_destroy(handle)
            self.handle = None


def _jacobi(diagonal, alpha, shift):
    alpha = complex(alpha)

    def M(y):
        out = torch.empty_like(y)
        check(LIB.he_vec_jacobi(y.numel(), _vp(diagonal), alpha.real, alpha.imag, float(shift), _vp(y), _vp(out),
                                _stream(y.device)), 'he_vec_jacobi')
        return out
    return M


@torch.no_grad()
def gmres(apply, b, preconditioner, x0=None, tol=1e-11, restart=32, max_restarts=10, flexible=False):
    """Right-preconditioned (flexible) GMRES (python/implicit.py:45-74) with the Krylov basis,
    CGS2 and all vector work on the device."""
    M = preconditioner if callable(preconditioner) else (lambda y: preconditioner * y)
    x = b.clone() if x0 is None else x0.clone()
    bnorm = norm(b)
    if bnorm == 0:
        return torch.zeros_like(b), {'iterations': 0, 'relative_residual': 0.}
    n = b.numel()
    ws = workspace(n, restart, b.device, flexible)
    stream = _stream(b.device)
    iterations = 0
    true = np.inf
    hostH = np.zeros((restart + 1, restart), complex)
    for _ in range(max_restarts):
        q0 = ws.vector(0)
        ax = apply(x)
        beta = ct.c_double()
        check(LIB.he_vec_residual_norm(n, _vp(b), _vp(ax), _vp(q0), ct.byref(beta), stream), 'residual')
        beta = beta.value
        if beta <= tol * bnorm:
            return x, {'iterations': iterations, 'relative_residual': beta / bnorm}
        check(LIB.he_krylov_scale(ws.handle, 0, 0, 1.0 / beta, stream), 'scale')
        check(LIB.he_krylov_reset(ws.handle, stream), 'reset')
        hostH[:] = 0
        column = np.zeros(2 * (restart + 1))
        read = 0   # Hessenberg columns read so far; the rest stay on the device until a check point
        for j in range(restart):
            z = M(ws.vector(j))
            if flexible:
                ws.vector(j, 1).copy_(z)
            ws.vector(j + 1).copy_(apply(z))
            iterations += 1
            check(LIB.he_krylov_orthogonalize(ws.handle, j, stream), 'orthogonalize')
            if (j + 1) % (2 if flexible else 4) != 0 and j + 1 != restart:
                check(LIB.he_krylov_normalize(ws.handle, j + 1, stream), 'normalize')
                continue
            # check point: read the pending columns; a breakdown (h < 1e-14) in one of them ends
            # the cycle there, with the same least squares as an immediate check would use
            for c in range(read, j + 1):
                check(LIB.he_krylov_hessenberg(ws.handle, c, c + 2, column.ctypes.data, stream), 'hessenberg')
                hostH[:c + 2, c] = column[:2 * (c + 2)].view(complex)
            read = j + 1
            broken = [c for c in range(j + 1) if hostH[c + 1, c].real < 1e-14]
            if broken:
                iterations -= j - broken[0]
                j = broken[0]
            hnorm = hostH[j + 1, j].real
            m = j + 1
            small = hostH[:m + 1, :m]
            rhs = np.zeros(m + 1, complex)
            rhs[0] = beta
            y = np.linalg.lstsq(small, rhs, rcond=None)[0]
            estimate = np.linalg.norm(rhs - small @ y)
            if estimate < tol * bnorm or hnorm < 1e-14 or m == restart:
                coef = np.ascontiguousarray(y, dtype=complex)
                if flexible:
                    candidate = x.clone()
                    check(LIB.he_krylov_combine_coef(ws.handle, 1, m, coef.ctypes.data, _vp(candidate), 1, stream),
                          'combine')
                else:
                    direction = torch.empty_like(x)
                    check(LIB.he_krylov_combine_coef(ws.handle, 0, m, coef.ctypes.data, _vp(direction), 0, stream),
                          'combine')
                    candidate = axpby(1, x, 1, M(direction))
                res = ct.c_double()
                check(LIB.he_vec_residual_norm(n, _vp(b), _vp(apply(candidate)), None, ct.byref(res), stream),
                      'true residual')
                true = res.value / bnorm
                if true <= tol:
                    return candidate, {'iterations': iterations, 'relative_residual': true}
                if hnorm < 1e-14 or m == restart:
                    x = candidate
                    break
            check(LIB.he_krylov_normalize(ws.handle, j + 1, stream), 'normalize')
    raise RuntimeError(f'GMRES did not converge: residual={true:.3e}, iterations={iterations}')


_DEVICE_SOLVES = [True]
_DEVICE_STEPS = [True]


def device_steps(flag=True):
    """Run a complex128 CF4 step as one C-ABI call (he_cf4_step: the four Pade solves, the
    state updates and the phases enqueued by the library) when the device solves apply (the
    default), or compose it here from :func:`device_gmres` calls; both run the same solves."""
    _DEVICE_STEPS[0] = bool(flag)


def device_solves(flag=True):
    """Run the Pade solves of pade_step / cf4_step as whole device GMRES solves
    (he_gmres_shifted: least squares, true-residual acceptance and restarts decided on the
    device, one status read per enqueued segment) when the engine and preconditioner allow
    it (the default), or through the host-driven :func:`gmres` loop."""
    _DEVICE_SOLVES[0] = bool(flag)


def _device_solver(engine, separable):
    """The engine/preconditioner pair the device GMRES can run: this package's engine with its
    own shifted operator, and the separable preconditioner or the Jacobi diagonal."""
    from .engine import B200Hamiltonian
    if not _DEVICE_SOLVES[0] or not isinstance(engine, B200Hamiltonian):
        return False
    if type(engine).apply_shifted is not B200Hamiltonian.apply_shifted:
        return False
    return separable is None or isinstance(separable, SeparablePreconditioner)


def device_gmres(engine, b, field, alpha, reference_energy, separable, shift, tol=1e-11, restart=32,
                 max_restarts=10, precision='complex128'):
    """GMRES (python/implicit.py:45-74) for (I + i alpha (H(field) - E_ref)) s = b, right
    preconditioned by ``separable`` (flexible when it is complex64) or, with ``separable``
    None, by the Jacobi diagonal 1 / (1 + i alpha (diag + shift)); precision 'complex64'
    applies H in complex64 (the inner solves of a mixed-precision Pade solve).  The whole
    solve runs on the device (he_gmres_shifted); results, iteration counts and the
    'GMRES did not converge' failure follow the reference's rules."""
    flexible = bool(getattr(separable, 'flexible', False))
    ws = workspace(b.numel(), restart, b.device, flexible)
    x = torch.empty_like(b)
    f = np.ascontiguousarray(field, dtype=np.float64)
    alpha = complex(alpha)
    iterations, residual = ct.c_int(), ct.c_double()
    code = HE_C64 if precision == 'complex64' else HE_C128
    status = LIB.he_gmres_shifted(ws.handle, engine.op.handle, separable.handle if separable is not None else None,
                                  None if separable is not None else _vp(engine.diagonal), _vp(b), _vp(x),
                                  f.ctypes.data, alpha.real, alpha.imag, float(reference_energy), float(shift),
                                  float(tol), int(restart), int(max_restarts), code, ct.byref(iterations),
                                  ct.byref(residual), _stream(b.device))
    if status == HE_ERR_NOCONV:
        raise RuntimeError(LIB.he_last_error().decode().split(' (')[0])
    check(status, 'he_gmres_shifted')
    return x, {'iterations': iterations.value, 'relative_residual': residual.value}


def device_cf4(engine, x, fields, dt, reference_energy, tol):
    """One complex128 CF4 step through he_cf4_step (python/implicit.py:91-109): fields are
    the vector potentials at t + C1 dt and t + C2 dt.  Raises the reference's 'GMRES did not
    converge' message when a solve fails, so :func:`cf4_step` halves dt as the reference does."""
    separable = getattr(engine, 'separable', None)
    flexible = bool(getattr(separable, 'flexible', False))
    restart = 16 if flexible else 32
    engine._check(x, torch.complex128)
    ws = workspace(x.numel(), restart, x.device, flexible)
    y = torch.empty_like(x)
    f = np.ascontiguousarray(fields, dtype=np.float64)
    iterations, residual = ct.c_int(), ct.c_double()
    status = LIB.he_cf4_step(ws.handle, engine.op.handle, separable.handle if separable is not None else None,
                             None if separable is not None else _vp(engine.diagonal), _vp(x), _vp(y), f.ctypes.data,
                             float(dt), float(reference_energy), float(getattr(engine, 'a2_coefficient', 1.)),
                             float(tol), restart, 10, ct.byref(iterations), ct.byref(residual), _stream(x.device))
    if status == HE_ERR_NOCONV:
        raise RuntimeError(LIB.he_last_error().decode().split(' (')[0])
    check(status, 'he_cf4_step')
    return y, {'linear_iterations': iterations.value, 'linear_residual': residual.value, 'dimension': 0,
               'residual_estimate': None}


INNER_TOLERANCE = 1e-5   # relative residual of each complex64 inner solve of a mixed Pade solve


def defect_corrected_solve(A, A32, b, M, tol, flexible, restart, corrections=8, inner=None, finish=None):
    """Solve A s = b to a complex128 relative residual <= tol by defect correction: each
    sweep solves A32 d = r by GMRES with the complex64 operator A32 (FP32 accumulation)
    to INNER_TOLERANCE, adds d to s and recomputes r = b - A s with the complex128
    operator.  Each sweep gains about five digits while that stays above the complex64
    operator's own error, so a 1e-11 solve takes two or three sweeps.  ``inner(r, tol)``,
    when given, replaces the host-driven inner GMRES (the device solver).

    When an inner solve cannot reach its tolerance, or a sweep gains less than a factor 10
    (the complex64 operator's own error reached), the remaining correction is solved in
    complex128 from the current s (``finish(r, tol)``, default: GMRES with A), so the solve
    still meets tol; info['fallback'] says so.  Raises the reference's 'GMRES did not
    converge' message when that also fails."""
    s = torch.zeros_like(b)
    r = b
    bnorm = norm(b)
    iterations, relative = 0, 1.
    if finish is None:
        finish = lambda rhs, t: gmres(A, rhs, M, tol=t, flexible=flexible, restart=restart)
    for sweep in range(corrections):
        try:
            if inner is not None:
                d, info = inner(r, max(INNER_TOLERANCE, tol))
            else:
                d, info = gmres(A32, r, M, tol=max(INNER_TOLERANCE, tol), flexible=flexible, restart=restart)
        except RuntimeError as error:
            if 'GMRES did not converge' not in str(error):
                raise
            break
        iterations += info['iterations']
        s = axpby(1, s, 1, d, out=s)
        r = axpby(1, b, -1, A(s))
        previous, relative = relative, norm(r) / bnorm
        if relative <= tol:
            return s, {'iterations': iterations, 'relative_residual': relative, 'corrections': sweep + 1,
                       'fallback': False}
        if relative > .1 * previous:
            break
    # complex128 solve of the remaining correction A d = r, to tol relative to ||b||
    rnorm = norm(r)
    d, info = finish(r, tol * bnorm / rnorm)
    iterations += info['iterations']
    s = axpby(1, s, 1, d, out=s)
    relative = norm(axpby(1, b, -1, A(s))) / bnorm
    if relative > tol * 1.01:
        raise RuntimeError(f'GMRES did not converge: residual={relative:.3e}, iterations={iterations}')
    return s, {'iterations': iterations, 'relative_residual': relative, 'corrections': sweep + 1, 'fallback': True}


@torch.no_grad()
def pade_step(engine, x, field, dt, reference_energy=0., tol=1e-11, precision='complex128'):
    """Two shifted solves (I + i alpha K) s = x, x <- 2 s - x, alpha = dt / (3 +- i sqrt 3)
    (python/implicit.py:76-89).  precision='mixed': each solve is a complex128 defect
    correction around complex64 inner GMRES solves (:func:`defect_corrected_solve`); the
    state, the residuals and the step stay complex128."""
    if precision not in ('complex128', 'mixed'):
        raise ValueError("precision must be 'complex128' or 'mixed'")
    a2 = getattr(engine, 'a2_coefficient', 1.)
    squared = a2 * sum(float(a) ** 2 for a in field)
    iterations, residual, corrections, fallbacks = 0, 0., 0, 0
    separable = getattr(engine, 'separable', None)
    flexible = getattr(separable, 'flexible', False)
    for root in (3 + 1j * SQRT3, 3 - 1j * SQRT3):
        alpha = dt / root

        def A(y, alpha=alpha):
            return engine.apply_shifted(y, field, alpha, reference_energy, velocity=True)

        if separable is not None:
            M = (lambda y, alpha=alpha: separable.apply(y, alpha, squared - reference_energy))
        else:
            M = _jacobi(engine.diagonal, alpha, squared - reference_energy)
        restart = 16 if flexible else 32
        on_device = _device_solver(engine, separable)
        if precision == 'mixed':
            def A32(y, alpha=alpha):
                return engine.apply_shifted(y.to(torch.complex64), field, alpha, reference_energy,
                                            velocity=True).to(torch.complex128)

            def inner(r, inner_tol, alpha=alpha):
                return device_gmres(engine, r, field, alpha, reference_energy, separable, squared - reference_energy,
                                    inner_tol, restart, precision='complex64')

            def finish(r, finish_tol, alpha=alpha):
                return device_gmres(engine, r, field, alpha, reference_energy, separable, squared - reference_energy,
                                    finish_tol, restart)
            s, info = defect_corrected_solve(A, A32, x, M, tol, flexible, restart, inner=inner if on_device else None,
                                             finish=finish if on_device else None)
            corrections += info['corrections']
            fallbacks += int(info['fallback'])
        elif on_device:
            s, info = device_gmres(engine, x, field, alpha, reference_energy, separable, squared - reference_energy,
                                   tol, restart)
        else:
            s, info = gmres(A, x, M, tol=tol, flexible=flexible, restart=restart)
        x = axpby(2, s, -1, x)
        iterations += info['iterations']
        residual = max(residual, info['relative_residual'])
    out = {'linear_iterations': iterations, 'linear_residual': residual}
    if precision == 'mixed':
        out.update(corrections=corrections, fallbacks=fallbacks)
    return x, out


@torch.no_grad()
def cf4_step(engine, x, avec, t, dt, reference_energy=0., tol=1e-11, depth=0, precision='complex128'):
    """Commutator-free 4th-order Magnus step (python/implicit.py:91-109); precision as in
    :func:`pade_step`."""
    fields = np.array([avec(t + C1 * dt), avec(t + C2 * dt)], float)
    iterations, residual, original = 0, 0., x
    extra = {}
    a2 = getattr(engine, 'a2_coefficient', 1.)
    try:
        separable = getattr(engine, 'separable', None)
        if precision == 'complex128' and _DEVICE_STEPS[0] and _device_solver(engine, separable):
            return device_cf4(engine, x, fields, dt, reference_energy, tol)
        for w in ((A2, A1), (A1, A2)):
            effective = 2 * np.einsum('a,aj->j', w, fields)
            correction = a2 * (np.dot(w, np.sum(fields ** 2, axis=1)) - .5 * np.dot(effective, effective))
            x, info = pade_step(engine, x, effective, dt / 2, reference_energy, tol, precision)
            phase = np.exp(-1j * dt * (correction + reference_energy / 2))
            x = axpby(phase, x, 0, x, out=x)
            iterations += info['linear_iterations']
            residual = max(residual, info['linear_residual'])
            for key in ('corrections', 'fallbacks'):
                if key in info:
                    extra[key] = extra.get(key, 0) + info[key]
        return x, {'linear_iterations': iterations, 'linear_residual': residual, 'dimension': 0,
                   'residual_estimate': None, **extra}
    except RuntimeError as error:
        if 'GMRES did not converge' not in str(error) or depth >= 6:
            raise
        x, a = cf4_step(engine, original, avec, t, dt / 2, reference_energy, tol / 2, depth + 1, precision)
        x, b = cf4_step(engine, x, avec, t + dt / 2, dt / 2, reference_energy, tol / 2, depth + 1, precision)
        return x, {'linear_iterations': a['linear_iterations'] + b['linear_iterations'],
                   'linear_residual': max(a['linear_residual'], b['linear_residual']), 'dimension': 0,
                   'residual_estimate': None, 'subdivided': True}
