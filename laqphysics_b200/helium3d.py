"""Two-electron Hamiltonian tables in product Y_lm channels (host setup).

Builds the arrays that the device H·psi consumes, with the same names, shapes,
dtypes and Fortran ordering as the reference's ``Helium`` (python/helium3d.py:12-50),
so an engine built from either object sees identical tables:

* ``ptr, col, tv``: CSR of the normalised radial kinetic matrix (zero based);
* ``diag[i,j,c]`` = u_{l1}(r_i) + u_{l2}(r_j), u_l = -2 cut/r + l(l+1)/(2 r^2);
  the two one-electron parts are also kept (``diag_parts``) so the device can
  form the diagonal on the fly instead of streaming it;
* ``rad[i,j,lam]`` = r_<^lam / r_>^(lam+1) * cut_i cut_j, with r_< / r_> picked by
  grid index (the ordered contour parameter, also on the ECS ray);
* Coulomb edges ``vptr, vc, vl, vcoef`` and dipole edges
  ``dptr, dc, de, dcoef(3, nd), ldiff`` per output channel.

``apply`` goes through this package's C-ABI ``tensor_apply`` (GPU, host pointers)
exactly as the reference's goes through its native library (python/helium3d.py:79-80).
"""
import numpy as np
from scipy.sparse.linalg import LinearOperator

from .angular import cartesian, channels, coulomb


def cutoff(x, inner, outer):
    """Smooth 1 -> 0 quintic switch between ``inner`` and ``outer``
    (the reference's python/tdse1d.py:18-21, used for the Coulomb cut)."""
    if not 0 < inner < outer:
        raise ValueError('0<cutoff_inner<cutoff_outer')
    u = np.clip((abs(x) - inner) / (outer - inner), 0, 1)
    return 1 - 10 * u ** 3 + 15 * u ** 4 - 6 * u ** 5


def one_electron_potential(r, cut, l):
    """Nuclear attraction plus centrifugal term for one electron of angular momentum l."""
    return -2 * cut / r + l * (l + 1) / (2 * r * r)


def multipole_table(r, cut, count):
    """rad[:, :, lam] for lam < count, Fortran ordered (python/helium3d.py:28-30)."""
    n = len(r)
    i, j = np.indices((n, n))
    lo = r[np.minimum(i, j)]
    hi = r[np.maximum(i, j)]
    weight = cut[:, None] * cut[None, :]
    return np.asfortranarray(np.stack([lo ** lam / hi ** (lam + 1) * weight for lam in range(count)], axis=2))


def separable_diagonal(d1, d2):
    """diag(i,j,c) = d1(i,c) + d2(j,c) as a Fortran-ordered (n, n, nc) array."""
    return np.asfortranarray(d1[:, None, :] + d2[None, :, :])


class Helium:
    """Product-basis two-electron Hamiltonian tables (python/helium3d.py:12-50)."""

    def __init__(self, grid, lmax=2, M=0, cutoff_radii=None):
        self.grid = grid
        self.r = np.asfortranarray(grid.r, dtype=complex)
        self.ch = channels(lmax, M)
        self.n = len(self.r)
        self.nc = len(self.ch)
        self.shape = (self.n, self.n, self.nc)
        self.size = int(np.prod(self.shape))
        T = grid.kinetic.tocsr()
        self.ptr = T.indptr.astype(np.int32)
        self.col = T.indices.astype(np.int32)
        self.tv = T.data.astype(complex)
        r = self.r
        self.cut = np.ones(self.n) if cutoff_radii is None else cutoff(r.real, *cutoff_radii)
        parts1 = [one_electron_potential(r, self.cut, l1) for (l1, _), _ in self.ch]
        parts2 = [one_electron_potential(r, self.cut, l2) for _, (l2, _) in self.ch]
        self.diag_parts = (np.asfortranarray(np.array(parts1).T), np.asfortranarray(np.array(parts2).T))
        self._diag = None
        self.rad = multipole_table(r, self.cut, 2 * lmax + 1)
        self._build_edges(2 * lmax + 1)
        self.exchange = np.array([self.ch.index((b, a)) for a, b in self.ch])

    @property
    def diag(self):
        """Full diagonal table diag(i,j,c) = u_{l1}(r_i) + u_{l2}(r_j), built on first use
        (the device forms it on the fly from ``diag_parts``)."""
        if self._diag is None:
            self._diag = separable_diagonal(*self.diag_parts)
        return self._diag

    def _build_edges(self, nlam):
        vp, vc, vl, vv = [0], [], [], []
        dp, dc, de, dv, dl = [0], [], [], [], []
        for bra in self.ch:
            for b, ket in enumerate(self.ch):
                for lam in range(nlam):
                    value = coulomb(bra, ket, lam)
                    if abs(value) > 1e-13:
                        vc.append(b); vl.append(lam); vv.append(value)
                for electron in (0, 1):
                    if bra[1 - electron] != ket[1 - electron]:
                        continue
                    value = cartesian(bra[electron], ket[electron])
                    if np.max(np.abs(value)) < 1e-13:
                        continue
                    dc.append(b); de.append(electron + 1); dv.append(value)
                    l, ll = bra[electron][0], ket[electron][0]
                    dl.append(l * (l + 1) - ll * (ll + 1))
            vp.append(len(vc)); dp.append(len(dc))
        for name, values in [('vptr', vp), ('vc', vc), ('vl', vl), ('dptr', dp), ('dc', dc), ('de', de)]:
            setattr(self, name, np.array(values, dtype=np.int32))
        self.vcoef = np.array(vv, complex)
        self.dcoef = np.asfortranarray(np.array(dv, complex).reshape(-1, 3).T)
        self.ldiff = np.array(dl, dtype=float)

    # --- surface flux (python/helium3d.py:52-77) ------------------------------------
    def prepare_surface(self, radius):
        """Rows of the exact discrete commutator [H, Theta(r2 - R)] (electron 2 leaves).

        ``surface_T`` = commutator rows, ``surface_P`` = i*comm*(r_b - r_a) (velocity
        gauge part); validation mirrors python/helium3d.py:52-67."""
        theta = (self.r.real > radius).astype(float)
        T = self.grid.kinetic.toarray()
        comm = T * (theta[None, :] - theta[:, None])
        self.surface_indices = np.flatnonzero(np.max(abs(comm), axis=1) > 1e-14)
        idx = self.surface_indices
        if not len(idx):
            raise ValueError('empty surface commutator')
        if np.any(abs(self.r[idx].imag) > 1e-12):
            raise ValueError('surface must be inside real grid')
        if np.any(abs(self.grid.weights[idx].imag) > 1e-12):
            raise ValueError('surface stencil touches the ECS bridge; extend the real domain')
        if np.any(self.cut[idx] > 1e-12):
            raise ValueError('Volkov surface stencil overlaps nonzero potential; increase R')
        self.surface_T = comm[idx, :]
        self.surface_P = (1j * comm * (self.r[None, :] - self.r[:, None]))[idx, :]
        return idx

    def flux(self, psi, field):
        """Host flux frame (n, n_s, nc); the device engine has its own fused version."""
        u = np.asarray(psi).reshape(self.shape, order='F')
        out = np.einsum('sj,ijc->isc', self.surface_T, u)
        for a in range(self.nc):
            for k in range(self.dptr[a], self.dptr[a + 1]):
                if self.de[k] != 2:
                    continue
                coef = np.dot(field, self.dcoef[:, k])
                if abs(coef) > 1e-15:
                    out[:, :, a] += coef * (u[:, :, self.dc[k]] @ self.surface_P.T)
        return out

    # --- operator ---------------------------------------------------------------------
    def apply(self, x, field=(0., 0., 0.), velocity=False):
        from .native import tensor_apply
        return tensor_apply(self, x, field, velocity)

    def operator(self, field=(0., 0., 0.), velocity=False):
        return LinearOperator((self.size, self.size), matvec=lambda x: self.apply(x, field, velocity), dtype=complex)

    def ground(self, tol=1e-10, method='coupled', cache_dir=None):
        if method != 'coupled':
            raise ValueError('only the coupled (total L=0) ground solve is provided')
        from .ground_s import GroundS
        return GroundS(self).solve(tol, cache_dir)

    def exchange_error(self, x):
        u = np.asarray(x).reshape(self.shape, order='F')
        return float(np.linalg.norm(u - u.transpose(1, 0, 2)[:, :, self.exchange]))
