"""Device backward propagation of the He+ channel functions chi_c(t) for tSURFF.

Replaces the reference's IonicAdjoint (python/ionic_adjoint.py:12-52) and its use by the
online surface preparation (python/streaming_surface.py:125-146): the channel functions
start from the dual final states and are propagated backward with the adjoint ionic
Hamiltonian H_ion(A)^dagger = H0^dagger + sum_a A_a P_a^dagger + |A|^2/2, by the same
CF4 Magnus + [2/2] Pade formula as the reference's sparse-LU SparseCF4
(python/implicit.py:111-123), here with right-preconditioned GMRES on the device (tolerance
1e-12, the reference's device setting).  All right-hand sides (one per distinct channel)
form one vector x[row, rhs]; the operator and the exact per-angular-block resolvent of
H0^dagger (the preconditioner) run in this package's kernels (csrc/ionic.cu).
"""
import ctypes as ct
from types import SimpleNamespace

import numpy as np
import torch
from scipy.linalg import eig, inv

from ._lib import LIB, check, ptr


def _vp(t):
    return ct.c_void_p(t.data_ptr())


def _stream(device):
    return ct.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class IonicAdjoint:
    a2_coefficient = 0.   # |A|^2/2 is a coefficient of its own (the identity plane)

    def __init__(self, ion, nrhs, device='cuda:0'):
        self.ion, self.device = ion, torch.device(device)
        self.n, self.na, self.nrhs = ion.n, ion.na, int(nrhs)
        self.ndof = self.n * self.na
        self.size = self.ndof * self.nrhs
        matrices = [m.conj().T.tocsr() for m in (ion.h0, *ion.P, ion.identity)]
        pattern = sum(abs(m) for m in matrices).tocsr()
        pattern.sort_indices()
        rows = np.repeat(np.arange(self.ndof), np.diff(pattern.indptr))
        cols = pattern.indices
        data = np.ascontiguousarray(np.array([np.asarray(m[rows, cols]).ravel() for m in matrices]), dtype=np.complex128)
        self._ptr = np.ascontiguousarray(pattern.indptr, dtype=np.int32)
        self._col = np.ascontiguousarray(cols, dtype=np.int32)
        self.nmat = len(matrices)
        handle = ct.c_void_p()
        with torch.cuda.device(self.device):
            check(LIB.he_ionic_create(ct.byref(handle), self.ndof, self.nrhs, self.nmat, len(cols), ptr(self._ptr),
                                      ptr(self._col), ptr(data)), 'he_ionic_create')
        self.handle = handle
        # exact resolvent of each angular block of H0^dagger (one eigendecomposition per l)
        S, Si, E, conditions = {}, {}, {}, {}
        for l in sorted({l for l, _ in ion.states}):
            i = next(k for k, (ll, _) in enumerate(ion.states) if ll == l)
            block = matrices[0][i * self.n:(i + 1) * self.n, i * self.n:(i + 1) * self.n].toarray()
            e, vec = eig(block)
            S[l], Si[l], E[l], conditions[l] = vec, inv(vec), e, float(np.linalg.cond(vec))
        if max(conditions.values()) > 1e12:
            raise ValueError('ill-conditioned ionic adjoint preconditioner')
        self.condition_numbers = conditions
        colmajor = lambda mats: np.ascontiguousarray(np.array([m.T for m in mats]), dtype=np.complex128)
        Sb = colmajor([S[l] for l, _ in ion.states])
        Sib = colmajor([Si[l] for l, _ in ion.states])
        Eb = np.ascontiguousarray(np.array([E[l] for l, _ in ion.states]), dtype=np.complex128)
        with torch.cuda.device(self.device):
            check(LIB.he_ionic_set_preconditioner(self.handle, self.na, self.n, ptr(Sb), ptr(Sib), ptr(Eb)),
                  'he_ionic_set_preconditioner')
        self.separable = SimpleNamespace(apply=self.precondition, flexible=False)
        self.diagonal = self.tensor(np.repeat(matrices[0].diagonal(), self.nrhs))

    def coefficients(self, field):
        """Field -> coefficients of the P planes and of the identity: (A_x, A_y, A_z, |A|^2/2)."""
        field = np.asarray(field, float)
        return np.r_[field, .5 * np.dot(field, field)]

    def tensor(self, x):
        return torch.as_tensor(np.array(x, dtype=np.complex128, copy=True), device=self.device).reshape(-1)

    def host(self, x):
        return x.detach().cpu().numpy().reshape(self.ndof, self.nrhs)

    def _apply(self, x, field, alpha, shift, shifted, out):
        if x.dtype != torch.complex128 or not x.is_contiguous() or x.numel() != self.size or x.device != self.device:
            raise ValueError(f'ionic state must be a contiguous complex128 tensor of {self.size} elements')
        coef = np.ascontiguousarray(np.r_[1., np.asarray(field, float)], dtype=np.float64)
        if coef.size != self.nmat:
            raise ValueError(f'{self.nmat - 1} field coefficients expected')
        y = torch.empty_like(x) if out is None else out
        alpha = complex(alpha)
        check(LIB.he_ionic_apply(self.handle, ptr(coef), coef.size, _vp(x), _vp(y), alpha.real, alpha.imag,
                                 float(shift), int(shifted), _stream(self.device)), 'he_ionic_apply')
        return y

    @torch.no_grad()
    def apply(self, x, field, velocity=True, out=None):
        """y = H(field) x with field = the coefficient vector of `coefficients`."""
        return self._apply(x, field, 0., 0., False, out)

    @torch.no_grad()
    def apply_shifted(self, x, field, alpha, reference_energy=0., velocity=True, out=None):
        """y = x + i alpha (H(field) - E_ref) x, the operator of one Pade solve."""
        return self._apply(x, field, alpha, reference_energy, True, out)

    @torch.no_grad()
    def precondition(self, x, alpha, shift):
        y = torch.empty_like(x)
        alpha = complex(alpha)
        check(LIB.he_ionic_precondition(self.handle, _vp(x), _vp(y), alpha.real, alpha.imag, float(shift),
                                        _stream(self.device)), 'he_ionic_precondition')
        return y

    def __del__(self):
        handle = getattr(self, 'handle', None)
        if handle is not None and handle.value:
            LIB.he_ionic_destroy(handle)
            self.handle = None


@torch.no_grad()
def channel_functions(ion, unique, avec, times, device='cuda:0', tol=1e-12):
    """chi at every time of the uniform grid `times` (device tensor (len(times), ndof,
    nrhs)): the dual final states at times[-1], then one backward CF4 step per interval
    (python/streaming_surface.py:197-205 with surface_stride 1)."""
    from .implicit import cf4_step
    engine = IonicAdjoint(ion, len(unique), device)
    times = np.asarray(times, float)
    dt = float(times[1] - times[0])
    chi = torch.empty((len(times), engine.ndof, engine.nrhs), dtype=torch.complex128, device=engine.device)
    state = engine.tensor(ion.dual_final_states(unique))
    chi[-1] = state.reshape(engine.ndof, engine.nrhs)
    coefficients = lambda s: engine.coefficients(avec(s))
    for i in range(len(times) - 1, 0, -1):
        state, _ = cf4_step(engine, state, coefficients, float(times[i]), -dt, 0., tol=tol)
        chi[i - 1] = state.reshape(engine.ndof, engine.nrhs)
    return chi
