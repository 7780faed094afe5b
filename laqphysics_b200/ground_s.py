"""Field-free singlet ground state in the compressed total-L=0 basis (host setup).

Same method as the reference's ``GroundS`` (python/ground_s.py:15-89): the S
state sum_m (-1)^(l-m) Y_lm Y_l,-m / sqrt(2l+1) reduces the problem to lmax+1
radial channels; LOBPCG is preconditioned by the exact separable inverse built
from the eigenvectors of each one-electron radial Hamiltonian.  The matvec runs in this
package's GPU kernels with the tables resident on the device for the whole solve.
"""
import hashlib
import os
from pathlib import Path

import numpy as np
from scipy.linalg import eigh
from scipy.sparse.linalg import LinearOperator, lobpcg
from sympy.physics.wigner import wigner_3j

from .helium3d import separable_diagonal


class GroundS:
    def __init__(self, h):
        self.parent = h
        self.n = h.n
        self.lmax = max(a[0] for a, _ in h.ch)
        self.nc = self.lmax + 1
        self.shape = (self.n, self.n, self.nc)
        self.size = int(np.prod(self.shape))
        for name in ('r', 'ptr', 'col', 'tv', 'rad'):
            setattr(self, name, getattr(h, name))
        pick = [h.ch.index(((l, 0), (l, 0))) for l in range(self.nc)]
        if hasattr(h, 'diag_parts'):
            self.diag_parts = tuple(np.asfortranarray(p[:, pick]) for p in h.diag_parts)
            self.diag = separable_diagonal(*self.diag_parts)
        else:
            self.diag = np.asfortranarray(np.stack([h.diag[:, :, c] for c in pick], axis=2))
        ptr, cols, orders, values = [0], [], [], []
        for l in range(self.nc):
            for j in range(self.nc):
                for k in range(abs(l - j), l + j + 1, 2):
                    c = (-1) ** (l + j) * np.sqrt((2 * l + 1) * (2 * j + 1)) * float(wigner_3j(l, j, k, 0, 0, 0)) ** 2
                    if abs(c) > 1e-14:
                        cols.append(j); orders.append(k); values.append(c)
            ptr.append(len(cols))
        self.vptr = np.array(ptr, np.int32)
        self.vc = np.array(cols, np.int32)
        self.vl = np.array(orders, np.int32)
        self.vcoef = np.array(values, complex)
        self.dptr = np.zeros(self.nc + 1, np.int32)
        self.dc = np.zeros(0, np.int32)
        self.de = np.zeros(0, np.int32)
        self.dcoef = np.empty((3, 0), complex, order='F')
        self.ldiff = np.zeros(0)

    def apply(self, x):
        """H x in the compressed basis on the GPU: the tables stay resident in one engine
        for the whole solve (only x and H x cross the bus per product)."""
        engine = getattr(self, '_engine', None)
        if engine is None:
            from .engine import B200Hamiltonian
            engine = self._engine = B200Hamiltonian(self, 'cuda:0')
        return engine.host(engine.apply(engine.state(x), (0., 0., 0.), False))

    def expand(self, x):
        u = np.asarray(x).reshape(self.shape, order='F')
        out = np.zeros(self.parent.shape, complex, order='F')
        for c, ((l, m), (j, mm)) in enumerate(self.parent.ch):
            if l == j and m == -mm:
                out[:, :, c] = (-1) ** (l - m) / np.sqrt(2 * l + 1) * u[:, :, l]
        return out.ravel(order='F')

    def _key(self, tol):
        digest = hashlib.sha256(b'helium-coupled-S-v1')
        for a in (self.r, self.parent.grid.weights, self.tv, self.col, self.ptr, self.parent.cut):
            digest.update(np.ascontiguousarray(a).tobytes())
        digest.update(str((self.lmax, tol)).encode())
        return digest.hexdigest()

    def solve(self, tol=1e-10, cache_dir=None, expand=True):
        if self.parent.grid.ecs_angle:
            raise ValueError('ground solve requires real grid')
        path = Path(cache_dir) / ('ground_' + self._key(tol) + '.npz') if cache_dir else None
        if path is not None and path.exists():
            data = np.load(path)
            small = data['state']
            return float(data['energy']), self.expand(small) if expand else small, float(data['residual'])
        r = self.r.real
        u = r * np.exp(-1.6875 * r) * np.sqrt(self.parent.grid.weights.real)
        x = np.zeros(self.shape)
        x[:, :, 0] = u[:, None] * u[None, :]
        op = LinearOperator((self.size, self.size), matvec=lambda v: self.apply(v).real, dtype=float)
        T = self.parent.grid.kinetic.toarray().real
        cut = self.parent.cut
        spectra, vectors = [], []
        for l in range(self.nc):
            e, U = eigh(T + np.diag(-2 * cut / r + l * (l + 1) / (2 * r * r)))
            spectra.append(e); vectors.append(U)
        shift = 2 * min(spectra[0]) - .5

        def precondition(y):
            y = np.asarray(y).reshape(self.shape, order='F')
            out = np.empty(self.shape)
            for l in range(self.nc):
                U, e = vectors[l], spectra[l]
                z = U.T @ y[:, :, l] @ U
                out[:, :, l] = U @ (z / (e[:, None] + e[None, :] - shift)) @ U.T
            return out.ravel(order='F')

        M = LinearOperator((self.size, self.size), matvec=precondition, dtype=float)
        E, v, history = lobpcg(op, x.reshape(-1, 1, order='F'), M=M, largest=False, tol=tol, maxiter=250,
                               retResidualNormsHistory=True)
        self.last_iterations = len(history)
        small = v[:, 0].astype(complex)
        res = float(np.linalg.norm(self.apply(small) - E[0] * small))
        if path is not None:
            path.parent.mkdir(parents=True, exist_ok=True)
            tmp = path.with_name(path.stem + f'.{os.getpid()}.tmp.npz')
            np.savez(tmp, state=small, energy=E[0], residual=res)
            os.replace(tmp, path)
        return float(E[0]), self.expand(small) if expand else small, res
