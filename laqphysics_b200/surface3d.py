"""Ionic (He+) channel set for channel-resolved tSURFF (host setup).

Same channel bookkeeping and operators as the reference's ``Ionic``
(python/surface3d.py:8-48): the inner-electron states are the sorted set of
first-electron (l, m) of the product channels (optionally restricted to the given m),
``h0`` is the block-diagonal ionic radial Hamiltonian, ``P`` the velocity-gauge
dipole couplings per Cartesian axis, and ``final_states`` / ``dual_final_states`` the
analytic bound states on the (complex) grid, the dual paired without conjugating the
radial argument (python/surface3d.py:37-42).
"""
import numpy as np
from scipy.sparse import block_diag, bmat, csr_matrix, diags, eye

from .angular import cartesian, radial_hydrogen


class Ionic:
    def __init__(self, h, magnetic_numbers=None):
        self.h = h
        self.states = sorted(set(a for a, b in h.ch if magnetic_numbers is None or a[1] in magnetic_numbers))
        self.n = h.n
        self.na = len(self.states)
        self.index = {a: i for i, a in enumerate(self.states)}
        T = h.grid.kinetic.tocsr()
        r = h.r
        self.h0 = block_diag([T + diags(-2 * h.cut / r + l * (l + 1) / (2 * r * r)) for l, _ in self.states],
                             format='csr')
        blocks = [[[csr_matrix((self.n, self.n), dtype=complex) if a == b else None for b in range(self.na)]
                   for a in range(self.na)] for _ in range(3)]
        base = T @ diags(r) - diags(r) @ T
        for a, (l, m) in enumerate(self.states):
            for b, (ll, mm) in enumerate(self.states):
                coef = cartesian((l, m), (ll, mm))
                if np.max(abs(coef)) < 1e-14:
                    continue
                pm = 1j * (base + diags((l * (l + 1) - ll * (ll + 1)) / (2 * r)))
                for axis in range(3):
                    if abs(coef[axis]) > 1e-14:
                        blocks[axis][a][b] = coef[axis] * pm
        self.P = [bmat(axis, format='csr') for axis in blocks]
        self.T = T
        self.identity = eye(self.n * self.na, format='csr')

    def final_states(self, labels):
        out = []
        for n, l, m in labels:
            z = np.zeros((self.na, self.n), complex)
            z[self.index[(l, m)]] = self.h.r * radial_hydrogen(n, l, self.h.r) * np.sqrt(self.h.grid.weights)
            out.append(z.ravel())
        return np.array(out).T

    def dual_final_states(self, labels):
        return self.final_states(labels).conj()

    def matrix(self, A):
        H = self.h0 + self.identity * np.dot(A, A) / 2
        for a, P in zip(A, self.P):
            if abs(a) > 0:
                H = H + a * P
        return H.tocsr()
