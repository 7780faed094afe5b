"""ORACLE (test infrastructure only): numpy restatement of the reference's Arnoldi
exponential propagator, python/propagate.py:6-50 (same algorithm as the device
version python/torch_backend.py:140-167).

exp(-i dt H) x is built in a Krylov space by classical Gram-Schmidt applied twice
(CGS2, :18-27); the small exponential expm(-i dt H_m)[:, 0] beta and the error
estimate |dt h_{m+1,m} c_m| are checked at happy breakdown (h < 1e-13) or whenever
j >= 3 and (j+1) % 4 == 0 or j+1 == maxdim (:29-31).  ``step`` evaluates H at the
midpoint t + dt/2 and halves dt recursively (depth <= 8) on non-convergence
(:41-50).
"""
import numpy as np
from scipy.linalg import expm


def exponential_action(apply, x, dt, tol=1e-11, maxdim=60):
    beta = np.linalg.norm(x)
    if beta == 0:
        return x.copy(), {'dimension': 0, 'residual_estimate': 0.}
    Q = np.empty((len(x), maxdim + 1), complex, order='F')
    H = np.zeros((maxdim + 1, maxdim), complex)
    Q[:, 0] = x / beta
    err = np.inf
    for j in range(maxdim):
        v = apply(Q[:, j])
        for _ in range(2):
            proj = Q[:, :j + 1].conj().T @ v
            H[:j + 1, j] += proj
            v = v - Q[:, :j + 1] @ proj
        H[j + 1, j] = np.linalg.norm(v)
        happy = abs(H[j + 1, j]) < 1e-13
        if happy or (j >= 3 and ((j + 1) % 4 == 0 or j + 1 == maxdim)):
            m = j + 1
            c = expm(-1j * dt * H[:m, :m])[:, 0] * beta
            err = abs(dt * H[m, m - 1] * c[-1])
            if happy or err < tol:
                return Q[:, :m] @ c, {'dimension': m, 'residual_estimate': float(err)}
        if j + 1 < maxdim:
            Q[:, j + 1] = v / H[j + 1, j]
    raise RuntimeError(f'Arnoldi did not converge: dim={maxdim}, dt={dt}, estimate={err:.3e}; reduce dt')


def step(apply_at, x, t, dt, tol=1e-11, maxdim=60, depth=0):
    try:
        return exponential_action(lambda y: apply_at(t + dt / 2, y), x, dt, tol, maxdim)
    except RuntimeError:
        if depth >= 8:
            raise
        y, a = step(apply_at, x, t, dt / 2, tol / 2, maxdim, depth + 1)
        y, b = step(apply_at, y, t + dt / 2, dt / 2, tol / 2, maxdim, depth + 1)
        return y, {'dimension': max(a['dimension'], b['dimension']),
                   'residual_estimate': a['residual_estimate'] + b['residual_estimate'], 'subdivided': True}


def exponential_action_fixed(apply, x, dt, m):
    """The same Krylov exponential with the dimension given instead of chosen: m CGS2
    Arnoldi vectors, y = Q_m expm(-i dt H_m)[:, 0] beta, and the error estimate
    |dt h_{m+1,m} c_m| the adaptive version would have compared with its tolerance (used to
    replay another implementation's step decisions on the same dimensions)."""
    beta = np.linalg.norm(x)
    Q = np.empty((len(x), m + 1), complex, order='F')
    H = np.zeros((m + 1, m), complex)
    Q[:, 0] = x / beta
    for j in range(m):
        v = apply(Q[:, j])
        for _ in range(2):
            proj = Q[:, :j + 1].conj().T @ v
            H[:j + 1, j] += proj
            v = v - Q[:, :j + 1] @ proj
        H[j + 1, j] = np.linalg.norm(v)
        if j + 1 < m:
            Q[:, j + 1] = v / H[j + 1, j]
    c = expm(-1j * dt * H[:m, :m])[:, 0] * beta
    return Q[:, :m] @ c, float(abs(dt * H[m, m - 1] * c[-1]))
