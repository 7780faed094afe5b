"""Bipolar (l1, l2, L, M) channels with both parities and every requested M (host setup).

Same basis, tables and change of basis as the reference's ``BipolarHelium``
(python/bipolar.py:35-122), the representation its production circular and pump-probe
inputs use: channels (l, j, L, m) for l, j <= lmax, |l - j| <= L <= min(l + j, total_Lmax),
every m in -L..L (or only m = M), unnatural parity included unless ``natural_parity``.

Construction (this package's own route): the bipolar channels are an exact Clebsch-Gordan
isometry U of the product channels (l m1)(j m2) with m1 + m2 = m,
U[(l m1)(j m2), (l j L m)] = (-1)^(l - j + m) sqrt(2L + 1) (l j L; m1 m2 -m), so every
operator is the product-basis operator projected as U^T A U: the Coulomb multipoles per
lambda and the three Cartesian dipole components of each electron.  They are re-emitted
as edge lists in the reference's order (per output channel: Coulomb edges by source, then
lambda; dipole edges of electron 1, then electron 2, by source) with its 1e-13 pruning, so
the device kernels consume the same tables (complex Cartesian dipole coefficients make the
field contraction complex for x/y polarisation).
"""
from types import SimpleNamespace

import numpy as np
from sympy.physics.wigner import wigner_3j

from .helium3d import Helium, one_electron_potential, separable_diagonal


class BipolarHelium:
    def __init__(self, grid, lmax=3, total_Lmax=3, M=None, cutoff_radii=None, natural_parity=False):
        product = Helium(grid, lmax, M=None, cutoff_radii=cutoff_radii)
        self.cutoff_radii = cutoff_radii
        self.grid, self.r, self.cut = grid, product.r, product.cut
        self.lmax, self.total_Lmax = lmax, total_Lmax
        self.basis = [(l, j, L, m) for l in range(lmax + 1) for j in range(lmax + 1)
                      for L in range(abs(l - j), min(l + j, total_Lmax) + 1)
                      if not natural_parity or (l + j - L) % 2 == 0
                      for m in range(-L, L + 1) if M is None or m == M]
        self.index = {c: i for i, c in enumerate(self.basis)}
        self.n, self.nc = product.n, len(self.basis)
        self.shape = (self.n, self.n, self.nc)
        self.size = int(np.prod(self.shape))
        for name in ('ptr', 'col', 'tv', 'rad'):
            setattr(self, name, getattr(product, name))
        U = np.zeros((product.nc, self.nc))
        for c, (l, j, L, m) in enumerate(self.basis):
            for a, ((l1, m1), (l2, m2)) in enumerate(product.ch):
                if l1 == l and l2 == j and m1 + m2 == m:
                    U[a, c] = (-1) ** (l - j + m) * np.sqrt(2 * L + 1) * float(wigner_3j(l, j, L, m1, m2, -m))
        if np.abs(U.T @ U - np.eye(self.nc)).max() > 1e-12:
            raise RuntimeError('bipolar transformation is not isometric')
        # rows: the product channels of the requested total M (python/bipolar.py:66-73)
        keep = [a for a, (x, y) in enumerate(product.ch) if M is None or x[1] + y[1] == M]
        self.transform = U[keep]
        self.diag_parts = (np.asfortranarray(np.array([one_electron_potential(self.r, self.cut, l)
                                                        for l, _, _, _ in self.basis]).T),
                           np.asfortranarray(np.array([one_electron_potential(self.r, self.cut, j)
                                                        for _, j, _, _ in self.basis]).T))
        self._diag = None
        self._project_edges(product, U)
        self.exchange = np.array([self.index[(j, l, L, m)] for l, j, L, m in self.basis])
        self.exchange_sign = np.array([(-1) ** (l + j - L) for l, j, L, _ in self.basis])
        self.uncoupled = SimpleNamespace(grid=grid, r=self.r, n=self.n, nc=len(keep),
                                         ch=[product.ch[a] for a in keep], cut=self.cut)
        self.uncoupled.prepare_surface = lambda radius: Helium.prepare_surface(self.uncoupled, radius)

    @property
    def diag(self):
        if self._diag is None:
            self._diag = separable_diagonal(*self.diag_parts)
        return self._diag

    def _project_edges(self, product, U):
        h = product
        nlam = h.rad.shape[2]
        V = np.zeros((nlam, h.nc, h.nc), complex)
        for a in range(h.nc):
            for k in range(h.vptr[a], h.vptr[a + 1]):
                V[h.vl[k], a, h.vc[k]] += h.vcoef[k]
        V = np.einsum('ap,lpq,qb->lab', U.T, V, U)
        D = np.zeros((2, 3, h.nc, h.nc), complex)    # electron, Cartesian component
        for a in range(h.nc):
            for k in range(h.dptr[a], h.dptr[a + 1]):
                D[h.de[k] - 1, :, a, h.dc[k]] += h.dcoef[:, k]
        D = np.einsum('ap,ecpq,qb->ecab', U.T, D, U)
        vp, vc, vl, vv = [0], [], [], []
        dp, dc, de, dv, dl = [0], [], [], [], []
        for a, bra in enumerate(self.basis):
            for b in range(self.nc):
                for lam in range(nlam):
                    if abs(V[lam, a, b]) > 1e-13:
                        vc.append(b); vl.append(lam); vv.append(V[lam, a, b].real)
            for e in range(2):
                for b, ket in enumerate(self.basis):
                    value = D[e, :, a, b]
                    if np.max(np.abs(value)) > 1e-13:
                        dc.append(b); de.append(e + 1); dv.append(value)
                        dl.append(bra[e] * (bra[e] + 1) - ket[e] * (ket[e] + 1))
            vp.append(len(vc)); dp.append(len(dc))
        for name, values in [('vptr', vp), ('vc', vc), ('vl', vl), ('dptr', dp), ('dc', dc), ('de', de)]:
            setattr(self, name, np.array(values, np.int32))
        self.vcoef = np.array(vv, complex)
        self.dcoef = np.asfortranarray(np.array(dv, complex).reshape(-1, 3).T)
        self.ldiff = np.array(dl, float)

    prepare_surface = Helium.prepare_surface
    flux = Helium.flux
    apply = Helium.apply
    operator = Helium.operator

    def expand(self, x):
        u = np.asarray(x).reshape(self.n * self.n, self.nc, order='F')
        return (u @ self.transform.T).ravel(order='F')

    def project(self, x):
        u = np.asarray(x).reshape(self.n * self.n, self.transform.shape[0], order='F')
        return (u @ self.transform).ravel(order='F')

    def ground(self, tol=1e-10, cache_dir=None):
        """Ground state from the total-L = 0 solve (python/bipolar.py:103-112): the
        (l, l, 0, 0) channels carry the compressed singlet solution."""
        from .ground_s import GroundS
        solver = GroundS(Helium(self.grid, self.lmax, M=0, cutoff_radii=self.cutoff_radii))
        E, g, res = solver.solve(tol, cache_dir, expand=False)
        small = g.reshape(solver.shape, order='F')
        out = np.zeros(self.shape, complex, order='F')
        for l in range(self.lmax + 1):
            if (l, l, 0, 0) in self.index:
                out[:, :, self.index[(l, l, 0, 0)]] = small[:, :, l]
        return E, out.ravel(order='F'), res

    def exchange_error(self, x):
        u = np.asarray(x).reshape(self.shape, order='F')
        swapped = u.transpose(1, 0, 2)[:, :, self.exchange] * self.exchange_sign[None, None, :]
        return float(np.linalg.norm(u - swapped))
