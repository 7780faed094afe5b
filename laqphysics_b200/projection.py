"""Clebsch-Gordan projection of product-channel tables onto coupled channels (host setup).

Both coupled bases of the engine, the M = 0 natural-parity (l1, l2, L) channels
(python/coupled_angular.py:13-82) and the bipolar (l1, l2, L, M) channels
(python/bipolar.py:35-122), are isometric images of the product channels
(l1 m1)(l2 m2).  Column c = (l1, l2, L, M) of the isometry is

    U[(l1 m1)(l2 m2), c] = (-1)^(l1 - l2 + M) sqrt(2L + 1) (l1 l2 L; m1 m2 -M),

a Clebsch-Gordan coefficient written through a 3j symbol.  Every channel-coupling table of
the product operator (Coulomb multipoles per lambda, the three Cartesian dipole components
of each electron) is a matrix A over product channels whose coupled form is U^T A U.  This
module builds U, scatters the product edge lists into those dense matrices, projects them in
one contraction each, and emits the non-zero couplings (|value| > 1e-13, the reference's
pruning) as the CSR-like edge lists the device kernels read.  The emission order is part of
the table format: Coulomb edges of one output channel by (source, lambda); dipole edges by
(source, electron) in the coupled M = 0 basis and by (electron, source) in the bipolar basis.
"""
from collections import defaultdict

import numpy as np
from sympy.physics.wigner import wigner_3j

from .helium3d import separable_diagonal

PRUNE = 1e-13


def isometry(product_channels, coupled_channels):
    """U (product x coupled) for coupled channels given as (l1, l2, L, M) tuples."""
    rows = defaultdict(list)
    for a, ((l1, m1), (l2, m2)) in enumerate(product_channels):
        rows[l1, l2].append((a, m1, m2))
    U = np.zeros((len(product_channels), len(coupled_channels)))
    for c, (l1, l2, L, M) in enumerate(coupled_channels):
        phase = (-1) ** (l1 - l2 + M) * np.sqrt(2 * L + 1)
        for a, m1, m2 in rows[l1, l2]:
            if m1 + m2 == M:
                U[a, c] = phase * float(wigner_3j(l1, l2, L, m1, m2, -M))
    return U


def check_isometry(U, what, tol):
    if np.abs(U.T @ U - np.eye(U.shape[1])).max() > tol:
        raise RuntimeError(f'{what}: the Clebsch-Gordan columns are not orthonormal')


def dense_couplings(product):
    """Product-basis coupling matrices: Coulomb V[lam, a, b] and dipole D[e, k, a, b]
    (electron e, Cartesian component k) from the product tables' edge lists."""
    nc, nlam = product.nc, product.rad.shape[2]
    rows = np.repeat(np.arange(nc), np.diff(product.vptr))
    V = np.zeros((nlam, nc, nc), complex)
    np.add.at(V, (product.vl, rows, product.vc), product.vcoef)
    rows = np.repeat(np.arange(nc), np.diff(product.dptr))
    D = np.zeros((2, 3, nc, nc), complex)
    for k in range(3):
        np.add.at(D[:, k], (product.de - 1, rows, product.dc), product.dcoef[k])
    return V, D


def _csr(rows, count):
    return np.concatenate(([0], np.cumsum(np.bincount(rows, minlength=count)))).astype(np.int32)


def project_tables(product, U, orbital, electron_major):
    """Projected edge lists for coupled channels.

    orbital[c] = (l1, l2) of coupled channel c; electron_major chooses the dipole order
    (electron, source) instead of (source, electron) within one output channel.
    """
    nc = U.shape[1]
    V, D = dense_couplings(product)
    V = np.einsum('pa,lpq,qb->abl', U, V, U)              # (output, source, lambda)
    D = np.einsum('pa,ekpq,qb->abek', U, D, U)            # (output, source, electron, xyz)
    a, b, lam = np.nonzero(np.abs(V) > PRUNE)
    tables = {'vptr': _csr(a, nc), 'vc': b.astype(np.int32), 'vl': lam.astype(np.int32),
              'vcoef': V[a, b, lam].real.astype(complex)}
    keep = np.abs(D).max(axis=3) > PRUNE                  # (output, source, electron)
    if electron_major:
        a, e, b = np.nonzero(keep.transpose(0, 2, 1))
    else:
        a, b, e = np.nonzero(keep)
    l_out = np.asarray(orbital)[a, e]
    l_in = np.asarray(orbital)[b, e]
    tables.update(dptr=_csr(a, nc), dc=b.astype(np.int32), de=(e + 1).astype(np.int32),
                  dcoef=np.asfortranarray(D[a, b, e].T), ldiff=(l_out * (l_out + 1) - l_in * (l_in + 1)).astype(float))
    return tables


class ProjectedChannels:
    """Shared behaviour of the coupled bases: tables live on the instance, the full
    diagonal is formed from its separable parts on first use, and states move between
    the coupled and product bases through the isometry."""

    @property
    def diag(self):
        if self._diag is None:
            self._diag = separable_diagonal(*self.diag_parts)
        return self._diag

    def _install(self, tables):
        for key, value in tables.items():
            setattr(self, key, value)

    def _columns(self, x, width):
        return np.asarray(x).reshape(self.n * self.n, width, order='F')

    def expand(self, x):
        """Coupled-basis state -> product-basis state (Fortran order)."""
        return (self._columns(x, self.nc) @ self.transform.T).ravel(order='F')

    def project(self, x):
        """Product-basis state -> coupled-basis state (Fortran order)."""
        return (self._columns(x, self.transform.shape[0]) @ self.transform).ravel(order='F')

    def exchange_error(self, x):
        """|| psi - P12 psi ||: r1 <-> r2 swap with the channel exchange and its (-1)^(l1+l2-L) sign."""
        u = np.asarray(x).reshape(self.shape, order='F')
        return float(np.linalg.norm(u - np.swapaxes(u, 0, 1)[:, :, self.exchange] * self.exchange_sign))

    def _embed_singlet(self, small, column_of_l):
        """Place the compressed total-L = 0 ground solution (one column per l) into the
        (l, l, L = 0) channels of this basis."""
        out = np.zeros(self.shape, complex, order='F')
        for l, column in column_of_l.items():
            out[:, :, column] = small[:, :, l]
        return out.ravel(order='F')
