"""Bipolar (l1, l2, L, M) channels with both parities and every requested M (host setup).

Same basis, tables and change of basis as the reference's ``BipolarHelium``
(python/bipolar.py:35-122), the representation its production circular and pump-probe
inputs use: channels (l, j, L, m) for l, j <= lmax, |l - j| <= L <= min(l + j, total_Lmax),
every m in -L..L (or only m = M), unnatural parity included unless ``natural_parity``.

Construction: the bipolar channels are an exact Clebsch-Gordan isometry of the product
channels (l m1)(j m2) with m1 + m2 = m, and every operator is the product-basis operator
projected through it (``projection.project_tables``): the Coulomb multipoles per lambda
and the three Cartesian dipole components of each electron, re-emitted in the bipolar
layout (per output channel: Coulomb edges by source, then lambda; dipole edges of
electron 1, then electron 2, by source), so the device kernels consume the same tables
(complex Cartesian dipole coefficients make the field contraction complex for x/y
polarisation).
"""
from types import SimpleNamespace

import numpy as np

from .helium3d import Helium, one_electron_potential
from .projection import ProjectedChannels, check_isometry, isometry, project_tables


class BipolarHelium(ProjectedChannels):
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
        U = isometry(product.ch, self.basis)
        check_isometry(U, 'bipolar channels', 1e-12)
        # rows: the product channels of the requested total M (python/bipolar.py:66-73)
        keep = [a for a, (x, y) in enumerate(product.ch) if M is None or x[1] + y[1] == M]
        self.transform = U[keep]
        self.diag_parts = (np.asfortranarray(np.array([one_electron_potential(self.r, self.cut, l)
                                                        for l, _, _, _ in self.basis]).T),
                           np.asfortranarray(np.array([one_electron_potential(self.r, self.cut, j)
                                                        for _, j, _, _ in self.basis]).T))
        self._diag = None
        self._install(project_tables(product, U, [c[:2] for c in self.basis], electron_major=True))
        self.exchange = np.array([self.index[(j, l, L, m)] for l, j, L, m in self.basis])
        self.exchange_sign = np.array([(-1) ** (l + j - L) for l, j, L, _ in self.basis])
        self.uncoupled = SimpleNamespace(grid=grid, r=self.r, n=self.n, nc=len(keep),
                                         ch=[product.ch[a] for a in keep], cut=self.cut)
        self.uncoupled.prepare_surface = lambda radius: Helium.prepare_surface(self.uncoupled, radius)

    prepare_surface = Helium.prepare_surface
    flux = Helium.flux
    apply = Helium.apply
    operator = Helium.operator

    def ground(self, tol=1e-10, cache_dir=None):
        """Ground state from the total-L = 0 solve (python/bipolar.py:103-112): the
        (l, l, 0, 0) channels carry the compressed singlet solution."""
        from .ground_s import GroundS
        solver = GroundS(Helium(self.grid, self.lmax, M=0, cutoff_radii=self.cutoff_radii))
        E, g, res = solver.solve(tol, cache_dir, expand=False)
        columns = {l: self.index[(l, l, 0, 0)] for l in range(self.lmax + 1) if (l, l, 0, 0) in self.index}
        return E, self._embed_singlet(g.reshape(solver.shape, order='F'), columns), res
