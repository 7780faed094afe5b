"""Coupled (l1, l2, L) channels of total M = 0 and natural parity (host setup).

Drop-in for the reference's ``CoupledHelium(uncoupled, total_Lmax)``
(python/coupled_angular.py:13-82): the same channel list (l1, l2 <= lmax, natural parity
l1 + l2 + L even, L <= total_Lmax), the same tables in the same format, the same
``transform``, ``exchange``/``exchange_sign``, ``expand``/``project``/``ground``/
``exchange_error``.  The tables are built by this package's projection module: the
product operator of ``uncoupled`` (an M = 0 ``Helium``) is projected through the
Clebsch-Gordan isometry in one contraction per table, and the edges are emitted in the
coupled layout (dipole edges ordered by source, then electron).
"""
import numpy as np

from .helium3d import Helium
from .projection import ProjectedChannels, check_isometry, isometry, project_tables


def natural_parity_channels(lmax, total_Lmax):
    """(l1, l2, L) with l1, l2 <= lmax, |l1 - l2| <= L <= min(l1 + l2, total_Lmax), l1 + l2 + L even."""
    out = []
    for l1 in range(lmax + 1):
        for l2 in range(lmax + 1):
            out += [(l1, l2, L) for L in range(abs(l1 - l2), min(l1 + l2, total_Lmax) + 1, 2)]
    return out


class CoupledHelium(ProjectedChannels):
    def __init__(self, uncoupled, total_Lmax):
        product = uncoupled
        total_m = {a[1] + b[1] for a, b in product.ch}
        if total_m != {0}:
            raise ValueError(f'the coupled basis is built from an M = 0 product basis (got total M {sorted(total_m)})')
        self.uncoupled = product
        self.lmax = max(l1 for (l1, _), _ in product.ch)
        self.total_Lmax = total_Lmax
        self.basis = natural_parity_channels(self.lmax, total_Lmax)
        self.n, self.nc = product.n, len(self.basis)
        self.shape = (self.n, self.n, self.nc)
        self.size = self.n * self.n * self.nc
        self.grid, self.r, self.cut = product.grid, product.r, product.cut
        self.ptr, self.col, self.tv, self.rad = product.ptr, product.col, product.tv, product.rad
        U = isometry(product.ch, [(l1, l2, L, 0) for l1, l2, L in self.basis])
        check_isometry(U, 'coupled M = 0 channels', 1e-11)
        self.transform = U
        # the diagonal is local in (l1, l2): take the parts of the (l1 0)(l2 0) product channel
        source = [product.ch.index(((l1, 0), (l2, 0))) for l1, l2, _ in self.basis]
        if hasattr(product, 'diag_parts'):
            self.diag_parts = tuple(np.asfortranarray(part[:, source]) for part in product.diag_parts)
            self._diag = None
        else:
            self._diag = np.asfortranarray(product.diag[:, :, source])
        self._install(project_tables(product, U, [c[:2] for c in self.basis], electron_major=False))
        where = {c: k for k, c in enumerate(self.basis)}
        self.exchange = np.array([where[l2, l1, L] for l1, l2, L in self.basis])
        self.exchange_sign = np.array([1 - 2 * ((l1 + l2 - L) & 1) for l1, l2, L in self.basis])

    prepare_surface = Helium.prepare_surface
    flux = Helium.flux

    def apply(self, x, field=(0., 0., 0.), velocity=False):
        """H·psi through the C-ABI; the M = 0 channels admit only a z field."""
        if max(abs(field[0]), abs(field[1])) > 1e-15:
            raise ValueError('an M = 0 coupled basis takes only a z field; use BipolarHelium for x/y fields')
        return Helium.apply(self, x, field, velocity)

    def ground(self, tol=1e-10, cache_dir=None):
        """Ground state of the compressed total-L = 0 problem, placed in the (l, l, 0) channels."""
        from .ground_s import GroundS
        solver = GroundS(self.uncoupled)
        energy, small, residual = solver.solve(tol, cache_dir, expand=False)
        columns = {l: self.basis.index((l, l, 0)) for l in range(self.lmax + 1)}
        return energy, self._embed_singlet(small.reshape(solver.shape, order='F'), columns), residual
