"""Coupled (l1, l2, L), M=0 channels with natural parity (host setup).

Same basis, tables and change-of-basis as the reference's ``CoupledHelium``
(python/coupled_angular.py:13-82): the coupled channels are an exact
Clebsch-Gordan isometry U of the product M=0 channels; Coulomb multipoles and
z dipoles are projected as U^T A U and re-emitted as edge lists with the
reference's 1e-13 pruning, so the device kernel consumes exactly the same
format for either basis.
"""
import numpy as np
from sympy.physics.wigner import wigner_3j

from .helium3d import Helium, separable_diagonal


class CoupledHelium:
    def __init__(self, uncoupled, total_Lmax):
        h = uncoupled
        self.uncoupled = h
        if any(a[1] + b[1] != 0 for a, b in h.ch):
            raise ValueError('coupled backend currently requires M=0')
        self.lmax = max(a[0] for a, _ in h.ch)
        self.total_Lmax = total_Lmax
        L1 = range(self.lmax + 1)
        self.basis = [(l, j, L) for l in L1 for j in L1
                      for L in range(abs(l - j), min(l + j, total_Lmax) + 1) if (l + j - L) % 2 == 0]
        self.n = h.n
        self.nc = len(self.basis)
        self.shape = (self.n, self.n, self.nc)
        self.size = int(np.prod(self.shape))
        self.grid, self.r, self.cut = h.grid, h.r, h.cut
        for name in ('ptr', 'col', 'tv', 'rad'):
            setattr(self, name, getattr(h, name))
        U = np.zeros((h.nc, self.nc))
        for c, (l, j, L) in enumerate(self.basis):
            for a, ((ll, m), (jj, mm)) in enumerate(h.ch):
                if l == ll and j == jj:
                    U[a, c] = (-1) ** (l - j) * np.sqrt(2 * L + 1) * float(wigner_3j(l, j, L, m, mm, 0))
        if np.linalg.norm(U.T @ U - np.eye(self.nc)) > 1e-11:
            raise RuntimeError('CG transformation is not isometric')
        self.transform = U
        zero_m = [h.ch.index(((l, 0), (j, 0))) for l, j, _ in self.basis]
        self._diag = None
        if hasattr(h, 'diag_parts'):
            self.diag_parts = tuple(np.asfortranarray(p[:, zero_m]) for p in h.diag_parts)
        else:
            self._diag = np.asfortranarray(np.stack([h.diag[:, :, c] for c in zero_m], axis=2))
        self._project_edges(h, U)
        self.exchange = np.array([self.basis.index((j, l, L)) for l, j, L in self.basis])
        self.exchange_sign = np.array([(-1) ** (l + j - L) for l, j, L in self.basis])

    @property
    def diag(self):
        if self._diag is None:
            self._diag = separable_diagonal(*self.diag_parts)
        return self._diag

    def _project_edges(self, h, U):
        nlam = h.rad.shape[2]
        V = []
        for lam in range(nlam):
            A = np.zeros((h.nc, h.nc), complex)
            for a in range(h.nc):
                for k in range(h.vptr[a], h.vptr[a + 1]):
                    if h.vl[k] == lam:
                        A[a, h.vc[k]] += h.vcoef[k]
            V.append(U.T @ A @ U)
        D = np.zeros((2, h.nc, h.nc), complex)
        for a in range(h.nc):
            for k in range(h.dptr[a], h.dptr[a + 1]):
                D[h.de[k] - 1, a, h.dc[k]] += h.dcoef[2, k]
        D = np.array([U.T @ A @ U for A in D])
        vp, vc, vl, vv = [0], [], [], []
        dp, dc, de, dv, dl = [0], [], [], [], []
        for a, (l, j, _) in enumerate(self.basis):
            for b, (ll, jj, _) in enumerate(self.basis):
                for lam, A in enumerate(V):
                    if abs(A[a, b]) > 1e-13:
                        vc.append(b); vl.append(lam); vv.append(A[a, b])
                for e in range(2):
                    if abs(D[e, a, b]) > 1e-13:
                        dc.append(b); de.append(e + 1); dv.append([0, 0, D[e, a, b]])
                        bra, ket = (l, j)[e], (ll, jj)[e]
                        dl.append(bra * (bra + 1) - ket * (ket + 1))
            vp.append(len(vc)); dp.append(len(dc))
        for name, values in [('vptr', vp), ('vc', vc), ('vl', vl), ('dptr', dp), ('dc', dc), ('de', de)]:
            setattr(self, name, np.array(values, np.int32))
        self.vcoef = np.array(vv, complex)
        self.dcoef = np.asfortranarray(np.array(dv, complex).reshape(-1, 3).T)
        self.ldiff = np.array(dl, float)

    prepare_surface = Helium.prepare_surface
    flux = Helium.flux

    def apply(self, x, field=(0., 0., 0.), velocity=False):
        if abs(field[0]) + abs(field[1]) > 1e-15:
            raise ValueError('M=0 coupled basis only supports z polarization')
        return Helium.apply(self, x, field, velocity)

    def expand(self, x):
        u = np.asarray(x).reshape(self.n * self.n, self.nc, order='F')
        return (u @ self.transform.T).ravel(order='F')

    def project(self, x):
        u = np.asarray(x).reshape(self.n * self.n, self.uncoupled.nc, order='F')
        return (u @ self.transform).ravel(order='F')

    def ground(self, tol=1e-10, cache_dir=None):
        from .ground_s import GroundS
        solver = GroundS(self.uncoupled)
        E, g, res = solver.solve(tol, cache_dir, expand=False)
        small = g.reshape(solver.shape, order='F')
        out = np.zeros(self.shape, complex, order='F')
        for l in range(self.lmax + 1):
            out[:, :, self.basis.index((l, l, 0))] = small[:, :, l]
        return E, out.ravel(order='F'), res

    def exchange_error(self, x):
        u = np.asarray(x).reshape(self.shape, order='F')
        swapped = u.transpose(1, 0, 2)[:, :, self.exchange] * self.exchange_sign[None, None, :]
        return float(np.linalg.norm(u - swapped))
