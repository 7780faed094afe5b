"""The backward recursion of laqphysics_b200/adjoint.py, restated with dense matrices on
the CPU: for a complex symmetric H(E) = H0 + E D the block exponential of
[[A, B], [0, A]] applied to conj(lambda) yields the costate step and the exact gradient of
the discrete Arnoldi-midpoint map; it must match central finite differences and scipy's
Frechet derivative of expm."""
import numpy as np
from scipy.linalg import expm, expm_frechet


def model(seed=3, n=12):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)) * 0.1
    H0 = (X + X.T) / 2                                # complex symmetric, not Hermitian
    Y = rng.normal(size=(n, n))
    D = (Y + Y.T) / 2
    psi0 = rng.normal(size=n) + 1j * rng.normal(size=n)
    psi0 /= np.linalg.norm(psi0)
    mask = (np.arange(n) >= n // 2).astype(float)
    return H0, D, psi0, mask


def forward(H0, D, psi0, E, dt, mask):
    psi = psi0.copy()
    states = [psi]
    for e in E:
        psi = expm(-1j * dt * (H0 + e * D)) @ psi
        states.append(psi)
    return float(np.vdot(psi, mask * psi).real), states


def gradient(H0, D, E, dt, mask, states):
    n = H0.shape[0]
    lam = mask * states[-1]
    g = np.zeros(len(E))
    for k in range(len(E) - 1, -1, -1):
        A, B = -1j * dt * (H0 + E[k] * D), -1j * dt * D
        M = np.block([[A, B], [np.zeros_like(A), A]])
        y = expm(M) @ np.concatenate([np.zeros(n), lam.conj()])
        top, bottom = y[:n], y[n:]
        g[k] = 2 * np.sum(top * states[k]).real
        lam = bottom.conj()
    return g


def test_block_exponential_gradient_matches_finite_differences():
    H0, D, psi0, mask = model()
    dt = 0.05
    E = np.array([0.1, -0.2, 0.05, 0.3, 0.0, -0.1])
    J, states = forward(H0, D, psi0, E, dt, mask)
    g = gradient(H0, D, E, dt, mask, states)
    h = 1e-6
    for k in range(len(E)):
        Ep, Em = E.copy(), E.copy()
        Ep[k] += h
        Em[k] -= h
        fd = (forward(H0, D, psi0, Ep, dt, mask)[0] - forward(H0, D, psi0, Em, dt, mask)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1e-3, abs(g).max()), (k, fd, g[k])


def test_block_top_is_the_frechet_derivative_and_conjugation_gives_the_adjoint():
    H0, D, psi0, mask = model(seed=5)
    dt, e = 0.07, 0.2
    A, B = -1j * dt * (H0 + e * D), -1j * dt * D
    v = psi0
    M = np.block([[A, B], [np.zeros_like(A), A]])
    y = expm(M) @ np.concatenate([np.zeros_like(v), v])
    np.testing.assert_allclose(y[:len(v)], expm_frechet(A, B, compute_expm=False) @ v, rtol=1e-12, atol=1e-13)
    # L(A, B)^H = L(A^H, B^H) = conj(L(A, B)) for complex symmetric A, B
    L = expm_frechet(A, B, compute_expm=False)
    np.testing.assert_allclose(L.conj().T, expm_frechet(A.conj().T, B.conj().T, compute_expm=False), atol=1e-13)
    np.testing.assert_allclose(L.conj().T, L.conj(), atol=1e-13)
