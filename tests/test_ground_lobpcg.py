"""Device-form LOBPCG of the ground-state solve (laqphysics_b200.ground_s), run on CPU
tensors: the iteration against dense eigh, and the batched separable preconditioner
against the reference's per-channel formula (python/ground_s.py:77-82)."""
import numpy as np
import torch


def test_lobpcg_finds_the_smallest_eigenpair():
    from laqphysics_b200.ground_s import lobpcg_device
    rng = np.random.default_rng(4)
    n = 300
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    evals = np.r_[-2.9, np.linspace(-1.5, 40., n - 1)]
    A = (Q * evals) @ Q.T
    A = (A + A.T) / 2
    At = torch.as_tensor(A)
    d = torch.as_tensor(np.diag(A) + 3.)                       # Jacobi-like preconditioner
    x0 = torch.as_tensor(rng.standard_normal(n))
    lam, x, history = lobpcg_device(lambda v: At @ v, lambda r: r / d, x0, 1e-10)
    assert abs(lam - evals[0]) < 1e-10
    assert history[-1] < 1e-10 and len(history) < 250
    assert abs(abs(float(x @ torch.as_tensor(Q[:, 0]))) - 1) < 1e-10


def test_separable_inverse_matches_per_channel_formula():
    from laqphysics_b200.ground_s import separable_inverse
    rng = np.random.default_rng(8)
    n, nc = 9, 3
    vectors, spectra = [], []
    for _ in range(nc):
        M = rng.standard_normal((n, n))
        e, U = np.linalg.eigh(M + M.T)
        vectors.append(U)
        spectra.append(e)
    shift = 2 * min(spectra[0]) - .5
    y = rng.standard_normal(n * n * nc)
    Y = y.reshape((n, n, nc), order='F')
    ref = np.empty((n, n, nc))
    for l in range(nc):
        U, e = vectors[l], spectra[l]
        z = U.T @ Y[:, :, l] @ U
        ref[:, :, l] = U @ (z / (e[:, None] + e[None, :] - shift)) @ U.T
    out = separable_inverse(spectra, vectors, shift, n, 'cpu')(torch.as_tensor(y)).numpy()
    np.testing.assert_allclose(out, ref.ravel(order='F'), rtol=1e-12, atol=1e-12)
