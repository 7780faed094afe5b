"""Mixed length/velocity gauge with a compact radial gauge function (device operator).

Same operator as the reference's MixedHamiltonian (python/mixed_gauge.py:73-117): with a
smooth switch f(r) (1 inside ``inner``, 0 beyond ``outer``) and q = r (1 - f), the state
psi_g = exp(i A.r f(r)) psi_V obeys, per electron,

    H0 + A.i[H0, q rhat] + E.r f rhat + 1/2 [A^2 (q/r)^2 + (q'^2 - (q/r)^2) (A.rhat)^2],

so the velocity gauge acts outside the switch (the tSURFF flux stays valid there) and the
length gauge inside.  The field-free part runs through the fused H·psi kernels; the gauge
terms (the [T, q] stencil with the dipole coefficients, q/(2 r^2) and r f dipole factors,
and the projected rhat_a rhat_b quadratic couplings) are added by one device kernel
(csrc/mixed.cu).  The field is the reference's 12-vector (A, E, A_a A_b) of
:func:`parameters`.
"""
import ctypes as ct

import numpy as np
import torch

from ._lib import LIB, check, ptr
from .angular import cartesian
from .engine import B200Hamiltonian, _stream

PAIRS = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))


def profile(r, inner, outer):
    """q = r (1 - f), r f, c0 = (1 - f)^2 and c2 = q'^2 - (1 - f)^2 on the grid, with the
    quintic smooth step f = 1 - 10 s^3 + 15 s^4 - 6 s^5, s = (Re r - inner) / (outer - inner)
    clipped to [0, 1] (inner = outer = 0: the velocity gauge everywhere)."""
    r = np.asarray(r)
    if inner == outer == 0:
        f = np.zeros(len(r))
        fp = np.zeros(len(r))
    else:
        if not 0 <= inner < outer:
            raise ValueError('mixed gauge needs 0 <= inner < outer')
        s = np.clip((r.real - inner) / (outer - inner), 0, 1)
        f = 1 - 10 * s ** 3 + 15 * s ** 4 - 6 * s ** 5
        fp = (-30 * s ** 2 + 60 * s ** 3 - 30 * s ** 4) / (outer - inner)
    q = r * (1 - f)
    qp = 1 - f - r * fp
    return q, r * f, (1 - f) ** 2, qp ** 2 - (1 - f) ** 2


def parameters(avec, efunc, t):
    """(A, E, A_a A_b for the six pairs, off-diagonal pairs doubled) at time t."""
    A = np.asarray(avec(t), float)
    E = np.asarray(efunc(t), float)
    return np.r_[A, E, [A[a] * A[b] * (1 if a == b else 2) for a, b in PAIRS]]


def angular_squares(states):
    """Projected rhat_a rhat_b on single-electron states (l, m), the sum over intermediate
    states running to l_max + 1 so that the projection is exact; (6, len, len)."""
    top = max(l for l, _ in states) + 1
    extended = [(l, m) for l in range(top + 1) for m in range(-l, l + 1)]
    N = np.array([[cartesian(a, b) for b in extended] for a in states]).transpose(2, 0, 1)
    squares = np.array([.5 * (N[a] @ N[b].conj().T + N[b] @ N[a].conj().T) for a, b in PAIRS])
    if np.max(np.abs(sum(squares[:3]) - np.eye(len(states)))) > 2e-12:
        raise RuntimeError('incomplete angular quadratic operator')
    return squares


def quadratic_edges(h):
    """Edges (per output channel: electron 1 then 2, by source) of the six projected
    rhat_a rhat_b of each electron in the channel basis of ``h`` (product, coupled or
    bipolar: built on the product channels and projected with ``h.transform``)."""
    base = getattr(h, 'uncoupled', h)
    states = sorted({a for a, _ in base.ch} | {b for _, b in base.ch})
    lookup = {s: i for i, s in enumerate(states)}
    one = angular_squares(states)
    U = getattr(h, 'transform', None)
    U = None if U is None else (U.toarray() if hasattr(U, 'toarray') else np.asarray(U))
    mats = []
    for e in range(2):
        Q = np.zeros((6, base.nc, base.nc), complex)
        for a, bra in enumerate(base.ch):
            for b, ket in enumerate(base.ch):
                if bra[1 - e] == ket[1 - e]:
                    Q[:, a, b] = one[:, lookup[bra[e]], lookup[ket[e]]]
        Q[np.abs(Q) < 1e-14] = 0
        if U is not None:
            Q = np.einsum('ap,kpq,qb->kab', U.T, Q, U)
        mats.append(Q)
    qptr, qc, qe, qv = [0], [], [], []
    for a in range(h.nc):
        for e in range(2):
            for b in range(h.nc):
                value = mats[e][:, a, b]
                if np.max(np.abs(value)) > 1e-13:
                    qc.append(b); qe.append(e + 1); qv.append(value)
        qptr.append(len(qc))
    return (np.array(qptr, np.int32), np.array(qc, np.int32), np.array(qe, np.int32),
            np.ascontiguousarray(np.array(qv, complex).reshape(-1, 6)))


class MixedB200Hamiltonian(B200Hamiltonian):
    """B200Hamiltonian in the mixed gauge: ``apply(x, field)`` with the 12-vector field of
    :func:`parameters` (``velocity`` is ignored: the gauge is the operator's)."""
    a2_coefficient = 0.   # the A_a A_b are coefficients of their own

    def __init__(self, h, device='cuda:0', inner=2., outer=4., **kwargs):
        super().__init__(h, device, **kwargs)
        q, F, c0, c2 = profile(h.r, inner, outer)
        r = np.asarray(h.r)
        c = lambda a: np.ascontiguousarray(np.asarray(a, complex))
        self._gauge = [c(q), c(.5 * q / (r * r)), c(F), c(c0), c(c2)]
        self._qptr, self._qc, self._qe, self._qcoef = quadratic_edges(h)
        with torch.cuda.device(self.device):
            check(LIB.he_set_mixed_gauge(self.op.handle, *(ptr(a) for a in self._gauge), len(self._qc),
                                         ptr(self._qptr), ptr(self._qc) if len(self._qc) else None,
                                         ptr(self._qe) if len(self._qc) else None,
                                         ptr(self._qcoef) if len(self._qc) else None), 'he_set_mixed_gauge')

    @torch.no_grad()
    def apply(self, x, field, velocity=True, out=None, precision=None):
        f = np.ascontiguousarray(field, dtype=np.float64)
        if f.shape != (12,):
            raise ValueError('mixed gauge requires A, E and six quadratic coefficients')
        if precision not in (None, 'complex128') or x.dtype != torch.complex128:
            raise ValueError('the mixed gauge runs in complex128')
        y = super().apply(x, (0., 0., 0.), False, out=out)      # field-free H psi
        check(LIB.he_apply_mixed_terms(self.op.handle, ct.c_void_p(x.data_ptr()), ct.c_void_p(y.data_ptr()),
                                       ptr(f), _stream(self.device)), 'he_apply_mixed_terms')
        return y

    @torch.no_grad()
    def apply_shifted(self, x, field, alpha, reference_energy=0., velocity=True, out=None):
        """x + i alpha (H(field) - E_ref) x (the operator of one Pade solve)."""
        y = self.apply(x, field)
        alpha = complex(alpha)
        a, b = 1 - 1j * alpha * reference_energy, 1j * alpha
        out = torch.empty_like(x) if out is None else out
        check(LIB.he_vec_axpby(x.numel(), a.real, a.imag, ct.c_void_p(x.data_ptr()), b.real, b.imag,
                               ct.c_void_p(y.data_ptr()), ct.c_void_p(out.data_ptr()), _stream(self.device)),
              'he_vec_axpby')
        return out
