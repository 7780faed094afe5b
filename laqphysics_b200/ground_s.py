"""Field-free singlet ground state in the compressed total-L=0 basis.

Same method as the reference's ``GroundS`` (python/ground_s.py:15-89): the S state
sum_m (-1)^(l-m) Y_lm Y_l,-m / sqrt(2l+1) reduces the problem to lmax+1 radial channels,
and LOBPCG is preconditioned by the exact separable inverse built from the eigenvectors of
each one-electron radial Hamiltonian.  Here the whole solve runs on the GPU: the matvec in
this package's H·psi kernels (tables resident in one engine), the separable inverse as
batched GEMMs over the channels, the LOBPCG vectors in device memory; only the 3 x 3
Rayleigh-Ritz problem of each iteration goes to the host.  method='eigsh' keeps the
reference's alternative (scipy Lanczos over the device matvec).
"""
import hashlib
import os
from pathlib import Path
from types import SimpleNamespace

import numpy as np
from scipy.linalg import eigh
from scipy.sparse.linalg import LinearOperator, eigsh
from sympy.physics.wigner import wigner_3j

from .helium3d import cutoff, multipole_table, one_electron_potential, separable_diagonal


def lobpcg_device(apply, precondition, x, tol, maxiter=250):
    """Smallest eigenpair of a symmetric operator by single-vector LOBPCG (Knyazev's
    locally optimal iteration, as scipy.sparse.linalg.lobpcg with one vector): each
    iteration takes the Rayleigh-Ritz pair of span{x, M r, p} with r = A x - lambda x and p
    the previous update direction.  The span is orthonormalised through the eigenvectors
    of its Gram matrix (directions below 1e-14 of the largest dropped), so a nearly
    dependent p is discarded instead of breaking the solve.  Converged when |r| < tol
    with |x| = 1 (scipy's residual tolerance).  apply/precondition map float64 device
    vectors; returns (lambda, x, residual norms)."""
    import torch
    x = x / torch.linalg.vector_norm(x)
    Ax = apply(x)
    lam = float(torch.dot(x, Ax))
    p = Ap = None
    history = []
    for _ in range(maxiter):
        r = Ax - lam * x
        history.append(float(torch.linalg.vector_norm(r)))
        if history[-1] < tol:
            break
        w = precondition(r)
        S = torch.stack([x, w] + ([p] if p is not None else []), 1)
        AS = torch.stack([Ax, apply(w)] + ([Ap] if p is not None else []), 1)
        scale = 1 / torch.linalg.vector_norm(S, dim=0)
        S, AS = S * scale, AS * scale
        GA, GB = (S.T @ AS).cpu().numpy(), (S.T @ S).cpu().numpy()
        GA, GB = (GA + GA.T) / 2, (GB + GB.T) / 2
        s, V = np.linalg.eigh(GB)
        keep = s > 1e-14 * s[-1]
        T = V[:, keep] / np.sqrt(s[keep])
        theta, C = np.linalg.eigh(T.T @ GA @ T)
        c = torch.as_tensor(T @ C[:, 0], dtype=S.dtype, device=S.device)
        x, Ax = S @ c, AS @ c
        p, Ap = S[:, 1:] @ c[1:], AS[:, 1:] @ c[1:]
        norm = torch.linalg.vector_norm(x)
        x, Ax = x / norm, Ax / norm
        lam = float(torch.dot(x, Ax))
    return lam, x, history


def separable_inverse(spectra, vectors, shift, n, device):
    """y -> sum over channels l of U_l [(U_l^T Y_l U_l) / (e_i + e_j - shift)] U_l^T on a
    float64 device vector in Fortran (i, j, l) order (the reference's LOBPCG preconditioner,
    python/ground_s.py:77-82), as batched GEMMs over the channels.  The bytes of Y_l seen as
    [l, j, i] are Y_l^T, and the map commutes with transposition (the divisor is symmetric),
    so it runs on that view unchanged."""
    import torch
    U = torch.as_tensor(np.array(vectors), dtype=torch.float64, device=device)          # (nc, n, n)
    D = torch.as_tensor(np.array([e[:, None] + e[None, :] - shift for e in spectra]), dtype=torch.float64,
                        device=device)
    shape = (len(vectors), n, n)

    def precondition(v):
        z = U.transpose(1, 2) @ v.view(shape) @ U
        return (U @ (z / D) @ U.transpose(1, 2)).reshape(-1)
    return precondition


class GroundS:
    @classmethod
    def from_grid(cls, grid, lmax, cutoff_radii=None):
        """Ground-only S representation built from the grid alone (python/ground_s.py:16-27):
        the lmax+1 compressed channels without the full operator; solve() then returns the
        compressed state."""
        r = np.asarray(grid.r)
        n = len(r)
        T = grid.kinetic.tocsr()
        cut = np.ones(n) if cutoff_radii is None else cutoff(r.real, *cutoff_radii)
        one = [one_electron_potential(r, cut, l) for l in range(lmax + 1)]
        parent = SimpleNamespace(
            n=n, nc=lmax + 1, shape=(n, n, lmax + 1), grid=grid, r=np.asfortranarray(r), cut=cut,
            ptr=T.indptr.astype(np.int32), col=T.indices.astype(np.int32), tv=T.data.astype(complex),
            rad=multipole_table(r, cut, 2 * lmax + 1), ch=[((l, 0), (l, 0)) for l in range(lmax + 1)],
            diag=np.asfortranarray(np.stack([u[:, None] + u[None, :] for u in one], axis=2)))
        result = cls(parent)
        result.compact_only = True
        return result

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

    def engine(self):
        """The device engine of the compressed operator (tables resident for the solve)."""
        engine = getattr(self, '_engine', None)
        if engine is None:
            from .engine import B200Hamiltonian
            engine = self._engine = B200Hamiltonian(self, 'cuda:0')
        return engine

    def apply(self, x):
        """H x in the compressed basis on the GPU (host vectors in and out)."""
        engine = self.engine()
        return engine.host(engine.apply(engine.state(x), (0., 0., 0.), False))

    def expand(self, x):
        if getattr(self, 'compact_only', False):
            return np.asarray(x).copy()
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

    def radial_spectra(self):
        """Eigenpairs of the one-electron radial Hamiltonian T + V_l of each compressed
        channel on the real grid, and the shift of the separable preconditioner
        (python/ground_s.py:71-76)."""
        T = self.parent.grid.kinetic.toarray().real
        r, cut = self.r.real, self.parent.cut
        spectra, vectors = [], []
        for l in range(self.nc):
            e, U = eigh(T + np.diag(-2 * cut / r + l * (l + 1) / (2 * r * r)))
            spectra.append(e)
            vectors.append(U)
        return spectra, vectors, 2 * min(spectra[0]) - .5

    def _lobpcg(self, x, tol):
        import torch
        engine = self.engine()
        precondition = separable_inverse(*self.radial_spectra(), self.n, engine.device)

        def apply(v):
            return engine.apply(v.to(torch.complex128), (0., 0., 0.), False).real.contiguous()

        start = torch.as_tensor(np.ascontiguousarray(x.ravel(order='F')), device=engine.device)
        E, v, history = lobpcg_device(apply, precondition, start, tol)
        self.last_iterations = len(history)
        return E, v.cpu().numpy()

    def solve(self, tol=1e-10, cache_dir=None, expand=True, method='lobpcg'):
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
        if method == 'lobpcg':
            E, v = self._lobpcg(x, tol)
        elif method == 'eigsh':
            op = LinearOperator((self.size, self.size), matvec=lambda y: self.apply(y).real, dtype=float)
            Es, vs = eigsh(op, k=1, which='SA', v0=x.ravel(order='F'), tol=tol, ncv=min(40, self.size - 1),
                           maxiter=20000)
            E, v = float(Es[0]), vs[:, 0]
        else:
            raise ValueError('unknown ground eigensolver')
        small = np.asarray(v).astype(complex)
        res = float(np.linalg.norm(self.apply(small) - E * small))
        if path is not None:
            path.parent.mkdir(parents=True, exist_ok=True)
            tmp = path.with_name(path.stem + f'.{os.getpid()}.tmp.npz')
            np.savez(tmp, state=small, energy=E, residual=res)
            os.replace(tmp, path)
        return float(E), self.expand(small) if expand else small, res
