"""Adjoint gradient of a propagation objective with respect to the field samples.

The reference has no gradient; this module adds one for the length-gauge Arnoldi
propagation of python/propagate.py:41-50 (midpoint field, fixed dt).  The forward map is

    psi_n = exp(-i dt H(E_n)) psi_{n-1},   E_n = E(t_{n-1} + dt/2),   n = 1..N,
    H(E) = H0 + E D  (length gauge along z, src/kernels.f90:147-152),
    E(t) = sum_k theta_k phi_k(t)  (piecewise-linear hat functions on K knots),

and the objective is J = <psi_N | P | psi_N> with P Hermitian: a real diagonal mask (the
probability of one electron beyond a radius, the population of a set of channels) or the
ion-channel yield :class:`ChannelYield` (He+ left in shell n with the other electron beyond
a radius).

Backward pass (exact for the discrete map, up to the Krylov tolerance):

* With A = -i dt H(E_n), B = -i dt D the derivative of the step map is the Frechet
  derivative L(A, B) of exp, read off the block exponential
  exp([[A, B], [0, A]]) [0; v] = [L(A, B) v; exp(A) v].
* H is complex symmetric on the exterior-scaled grid (H^T = H, checked by
  :func:`check_complex_symmetric`), so A^dagger = conj(A), B^dagger = conj(B), and one block
  exponential applied to conj(lambda_n) gives both the costate step
  lambda_{n-1} = exp(A^dagger) lambda_n (bottom block, conjugated back) and the
  gradient term dJ/dE_n = 2 Re <L(A^dagger, B^dagger) lambda_n | psi_{n-1}> (top block).
* lambda_N = P psi_N (dJ = 2 Re <P psi_N | d psi_N> for Hermitian P);
  dJ/dtheta = sum_n (dJ/dE_n) phi_k(t_{n-1} + dt/2).
* The block exponential is one fused device solve (he_expv_field_derivative): per Krylov
  vector one batched apply of the two halves (H u, H w) and one dipole pass (D w), so a
  backward step costs about two forward steps.
* Every forward state stays in device memory when the states fit a quarter of the free
  memory (no recompute); otherwise states are kept every `checkpoint` steps and each
  segment is recomputed forward before its backward sweep.

:class:`AdjointObjective` wraps the pair as a ``torch.autograd.Function``.
"""
import numpy as np
import torch

from .angular import radial_hydrogen
from .torch_backend import FieldOperator, exponential_action, field_derivative_action


class ChannelYield:
    """P = sum_c |phi_{n, l1(c)}><phi_{n, l1(c)}| (electron 1) x Theta(r2 > radius): the
    probability of finding He+ in shell n (every l < n that the channels carry) with the
    second electron beyond `radius`, the box form of an ion-channel yield.  phi_{n l} is the
    hydrogenic Z = 2 radial function on the grid (r R_nl(r) sqrt(w), normalised on the grid);
    channels whose electron-1 momentum has no state in shell n contribute nothing."""

    def __init__(self, h, device, shell=2, radius=8.):
        r, w = np.asarray(h.r), np.asarray(h.grid.weights)
        phi = {}
        for l in range(shell):
            v = r * radial_hydrogen(shell, l, r, 2.0) * np.sqrt(w)
            phi[l] = v / np.linalg.norm(v)
        labels = [c[0] for c in h.basis] if hasattr(h, 'basis') else [a[0] for a, _ in h.ch]
        Phi = np.array([phi[l] if l in phi else np.zeros(h.n, complex) for l in labels])
        self.n, self.nc = h.n, h.nc
        self.Phi = torch.as_tensor(Phi, dtype=torch.complex128, device=device)            # (nc, n) over r1
        self.outer = torch.as_tensor((np.asarray(r).real > radius).astype(float), dtype=torch.complex128,
                                     device=device)                                          # over r2

    def __call__(self, psi):
        """P psi for a Fortran-order state psi(i, j, c) (viewed as u[c, j, i])."""
        u = psi.reshape(self.nc, self.n, self.n)
        a = torch.einsum('ci,cji->cj', self.Phi.conj(), u) * self.outer[None, :]
        return torch.einsum('ci,cj->cji', self.Phi, a).reshape(-1)


def hat_weights(knots, t):
    """Values of the piecewise-linear hat functions on `knots` at times t: (len(t), K)."""
    knots = np.asarray(knots, float)
    t = np.asarray(t, float)
    W = np.zeros((t.size, knots.size))
    idx = np.clip(np.searchsorted(knots, t, side='right') - 1, 0, knots.size - 2)
    frac = (t - knots[idx]) / (knots[idx + 1] - knots[idx])
    inside = (t >= knots[0]) & (t <= knots[-1])
    rows = np.arange(t.size)
    W[rows[inside], idx[inside]] = 1 - frac[inside]
    W[rows[inside], idx[inside] + 1] = frac[inside]
    return W


def check_complex_symmetric(engine, seed=0, tol=1e-10):
    """x^T H y == y^T H x for random x, y (both field 0 and field 1): the property the
    conjugation trick of the backward pass rests on.  Returns the relative defect."""
    rng = np.random.default_rng(seed)
    worst = 0.
    for field in ((0., 0., 0.), (0., 0., 1.)):
        x = engine.state(rng.normal(size=engine.size) + 1j * rng.normal(size=engine.size))
        y = engine.state(rng.normal(size=engine.size) + 1j * rng.normal(size=engine.size))
        a = torch.sum(x * engine.apply(y, field, False))
        b = torch.sum(y * engine.apply(x, field, False))
        worst = max(worst, float(abs(a - b) / max(abs(a), 1e-300)))
    if worst > tol:
        raise ValueError(f'H is not complex symmetric (relative defect {worst:.2e}); the adjoint needs H^T = H')
    return worst


class Propagation:
    """Fixed-step length-gauge Arnoldi propagation of one state under a sampled field.

    engine: B200Hamiltonian; psi0: initial state (numpy or device tensor); dt, steps;
    knots: K sample times of E(t); mask: the objective's P, a real diagonal (numpy,
    engine.size) or a callable psi -> P psi on the device (Hermitian, e.g. ChannelYield);
    tol/maxdim: Krylov controls (no dt halving: the gradient is that of this exact map,
    so a step that does not converge raises); checkpoint: steps between kept states (None:
    every state when all fit a quarter of the free device memory, else 64)."""

    def __init__(self, engine, psi0, dt, steps, knots, mask, tol=1e-13, maxdim=30, checkpoint=None):
        self.engine, self.dt, self.steps = engine, float(dt), int(steps)
        self.tol, self.maxdim = float(tol), int(maxdim)
        if checkpoint is None:
            free, _ = torch.cuda.mem_get_info(engine.device)
            checkpoint = 1 if (self.steps + 1) * engine.size * 16 <= free // 4 else 64
        self.checkpoint = max(1, int(checkpoint))
        self.psi0 = psi0 if torch.is_tensor(psi0) else engine.state(psi0)
        self.knots = np.asarray(knots, float)
        self.tmid = self.dt * (np.arange(self.steps) + 0.5)
        self.W = hat_weights(self.knots, self.tmid)                       # (steps, K)
        if callable(mask):
            self.P = mask
        else:
            diagonal = torch.as_tensor(np.asarray(mask, float), device=engine.device).to(torch.complex128)
            self.P = lambda psi: diagonal * psi

    def fields(self, theta):
        return self.W @ np.asarray(theta, float)

    def _step(self, psi, e):
        op = FieldOperator(self.engine, (0., 0., float(e)), velocity=False)
        y, info = exponential_action(op, psi, self.dt, self.tol, self.maxdim)
        return y

    def forward(self, theta, keep=True):
        """J(theta); keeps the checkpoint states when `keep`."""
        E = self.fields(theta)
        psi = self.psi0.clone()
        self._checkpoints = {0: psi.clone()} if keep else None
        for n in range(self.steps):
            psi = self._step(psi, E[n])
            if keep and (n + 1) % self.checkpoint == 0 and n + 1 < self.steps:
                self._checkpoints[n + 1] = psi            # each step returns a new tensor
        self._final = psi
        self._E = E
        return float(torch.sum(psi.conj() * self.P(psi)).real)

    def _block_apply(self, e):
        """z = [u; w] -> [H(E) u + D w; H(E) w] with D w = H(E+1) w - H(E) w, as a callable
        for the host-looped exponential_action (the form the fused derivative solve is
        tested against); the result buffer is reused (the caller copies it)."""
        from .implicit import axpby
        engine, size = self.engine, self.engine.size
        fields = np.array([[0., 0., e], [0., 0., e]])
        shifted = (0., 0., e + 1.)
        pair = torch.empty((2, size), dtype=torch.complex128, device=engine.device)
        out = torch.empty(2 * size, dtype=torch.complex128, device=engine.device)
        top, bottom = out[:size], out[size:]

        def apply(z):
            engine.apply_batched(z.view(2, size), fields, False, out=pair)
            engine.apply(z[size:], shifted, False, out=top)
            axpby(1, top, -1, pair[1], out=top)            # D w
            axpby(1, pair[0], 1, top, out=top)             # H(E) u + D w
            bottom.copy_(pair[1])
            return out
        return apply

    def gradient(self):
        """dJ/dtheta for the last forward(theta, keep=True) call."""
        if self._checkpoints is None:
            raise RuntimeError('run forward(theta, keep=True) first')
        size, E = self.engine.size, self._E
        lam = self.P(self._final)                                      # dJ/dpsi_N (up to the factor 2 in Re)
        gE = np.zeros(self.steps)
        starts = sorted(self._checkpoints)
        for s in reversed(starts):
            stop = min(s + self.checkpoint, self.steps)
            states = [self._checkpoints[s]]                            # psi_s .. psi_{stop-1}
            for n in range(s, stop - 1):
                states.append(self._step(states[-1], E[n]))
            for n in range(stop - 1, s - 1, -1):                       # step n maps psi_n -> psi_{n+1}
                z = torch.cat([torch.zeros_like(lam), lam.conj()])
                y, _ = field_derivative_action(self.engine, z, (0., 0., float(E[n])), (0., 0., 1.), self.dt,
                                               self.tol, self.maxdim)
                top, bottom = y[:size], y[size:]
                gE[n] = 2.0 * float(torch.sum(top * states[n - s]).real)
                lam = bottom.conj()
        return self.W.T @ gE


class AdjointObjective(torch.autograd.Function):
    """theta (CPU float64 tensor of knot values) -> J, with the adjoint gradient."""

    @staticmethod
    def forward(ctx, theta, propagation):
        J = propagation.forward(theta.detach().cpu().numpy(), keep=True)
        ctx.propagation = propagation
        return theta.new_tensor(J)

    @staticmethod
    def backward(ctx, grad_out):
        g = ctx.propagation.gradient()
        return grad_out * torch.as_tensor(g, dtype=grad_out.dtype), None
