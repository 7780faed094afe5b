"""Adjoint gradient of a length-gauge propagation on the GPU (laqphysics_b200.adjoint)
against central finite differences of the same device propagation.

Tolerance: |grad - FD| <= 1e-6 relative to the largest gradient component (the bar of the
adjoint form), with the Krylov tolerance at 1e-13 so that the forward map is smooth at the
finite-difference step h = 1e-5.  The FP64 reference gradient is the same central
difference taken on the CPU oracle's propagation (numpy Arnoldi + C tensor_apply), so the
device gradient is checked against a path that shares no device code."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'


def setup(steps=24, checkpoint=8, with_tables=False):
    from laqphysics_b200.adjoint import Propagation, check_complex_symmetric
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.workloads import coupled, seeded_state
    h = coupled(np.linspace(0, 12, 7), 6, 1, 1, ecs_angle=.3, tail=8, cutoff_radii=(8., 10.))
    engine = B200Hamiltonian(h, DEVICE)
    check_complex_symmetric(engine)
    psi0 = seeded_state(h.size, 11)
    psi0 /= np.linalg.norm(psi0)
    r = np.asarray(h.r).real
    outer = (r > 6.0).astype(float)
    mask = np.broadcast_to(outer[None, :, None], (h.n, h.n, h.nc)).ravel(order='F')   # electron 2 beyond 6 a.u.
    dt = 0.05
    knots = np.linspace(0, steps * dt, 6)
    prop = Propagation(engine, psi0, dt, steps, knots, mask, tol=1e-13, maxdim=30, checkpoint=checkpoint)
    theta = np.array([0.05, -0.08, 0.12, 0.02, -0.06, 0.09])
    return (prop, theta, h, psi0, mask) if with_tables else (prop, theta)


def test_adjoint_gradient_matches_central_differences():
    prop, theta = setup()
    J = prop.forward(theta)
    g = prop.gradient()
    h = 1e-5
    scale = np.abs(g).max()
    assert scale > 0 and np.isfinite(J)
    for k in range(len(theta)):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (prop.forward(tp, keep=False) - prop.forward(tm, keep=False)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * scale, (k, fd, g[k])


def test_autograd_function_and_checkpoint_length_do_not_change_the_gradient():
    from laqphysics_b200.adjoint import AdjointObjective
    prop, theta = setup(checkpoint=5)
    t = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    J = AdjointObjective.apply(t, prop)
    J.backward()
    prop2, _ = setup(checkpoint=64)
    prop2.forward(theta)
    np.testing.assert_allclose(t.grad.numpy(), prop2.gradient(), rtol=1e-10, atol=1e-14)
    prop3, _ = setup(checkpoint=None)            # every state resident: no recompute
    assert prop3.checkpoint == 1
    prop3.forward(theta)
    np.testing.assert_allclose(prop3.gradient(), prop2.gradient(), rtol=1e-10, atol=1e-14)


def test_dipole_pass_is_the_field_difference_of_h():
    """he_apply_dipole adds (direction . d) psi = H(f + direction) psi - H(f) psi (length gauge)."""
    import ctypes as ct
    from laqphysics_b200._lib import LIB, check, ptr
    from laqphysics_b200.engine import _stream
    from laqphysics_b200.workloads import seeded_state
    prop, _ = setup()
    engine = prop.engine
    x = engine.state(seeded_state(engine.size, 3))
    f, d = np.array([0.01, -0.02, 0.03]), np.array([0.3, -0.5, 1.0])
    diff = engine.apply(x, f + d, False) - engine.apply(x, f, False)
    base = torch.randn(engine.size, dtype=torch.complex128, device=DEVICE)
    out = base.clone()
    check(LIB.he_apply_dipole(engine.op.handle, ct.c_void_p(x.data_ptr()), ct.c_void_p(out.data_ptr()),
                              ptr(np.ascontiguousarray(d)), _stream(engine.device)), 'he_apply_dipole')
    err = torch.linalg.norm(out - base - diff) / torch.linalg.norm(diff)
    assert err < 1e-12, float(err)


def test_fused_derivative_solve_matches_host_block_exponential():
    """he_expv_field_derivative (fused block Arnoldi: batched apply + dipole pass) against the
    host-looped Arnoldi over the explicit block operator [[H, H(E+1) - H(E)], [0, H]]."""
    from laqphysics_b200.torch_backend import exponential_action, field_derivative_action
    from laqphysics_b200.workloads import seeded_state
    prop, _ = setup()
    engine, size = prop.engine, prop.engine.size
    z = torch.cat([engine.state(seeded_state(size, 5)), engine.state(seeded_state(size, 6))])
    E = 0.07
    ref, info_ref = exponential_action(prop._block_apply(E), z, prop.dt, 1e-13, 30)
    ref = ref.clone()
    for _ in range(2):                      # the second call replays the captured graph
        y, info = field_derivative_action(engine, z, (0., 0., E), (0., 0., 1.), prop.dt, 1e-13, 30)
        err = torch.linalg.norm(y - ref) / torch.linalg.norm(ref)
        assert err < 1e-11, float(err)
        assert info['dimension'] <= info_ref['dimension']


def test_adjoint_gradient_matches_oracle_fp64_gradient():
    """Device adjoint gradient against central differences of the CPU oracle propagation
    (the reference's Arnoldi restated in numpy over the C H·psi), h = 1e-5."""
    from oracle import arnoldi, cpu
    prop, theta, h, psi0, mask = setup(with_tables=True)
    prop.forward(theta)
    g = prop.gradient()
    tables = cpu.host_tables(h)

    def objective(th):
        E = prop.fields(th)
        x = psi0.copy()
        for n in range(prop.steps):
            x, _ = arnoldi.exponential_action(
                lambda y, e=E[n]: cpu.tensor_apply(h, y, (0., 0., e), False, tables=tables), x, prop.dt, 1e-13, 30)
        return float(np.sum(mask * np.abs(x) ** 2))

    from threadpoolctl import threadpool_limits
    step = 1e-5
    with threadpool_limits(limits=1, user_api='blas'):   # OpenMP in the C oracle, BLAS single-threaded
        ref = np.array([(objective(theta + step * e) - objective(theta - step * e)) / (2 * step)
                        for e in np.eye(len(theta))])
    assert np.abs(ref).max() > 0
    assert np.abs(g - ref).max() <= 1e-6 * np.abs(ref).max(), (g, ref)


def test_channel_yield_gradient_matches_device_and_oracle_differences():
    """Objective = He+(n = 2) yield with the second electron beyond 6 a.u. (a Hermitian,
    non-diagonal P): adjoint gradient against central differences of the device propagation
    and of the CPU oracle propagation (h = 1e-5), 1e-6 of the largest component."""
    from threadpoolctl import threadpool_limits
    from oracle import arnoldi, cpu
    from laqphysics_b200.adjoint import ChannelYield, Propagation
    prop0, theta, h, psi0, _ = setup(with_tables=True)
    P = ChannelYield(h, DEVICE, shell=2, radius=6.)
    prop = Propagation(prop0.engine, psi0, prop0.dt, prop0.steps, prop0.knots, P, tol=1e-13, maxdim=30, checkpoint=8)
    J = prop.forward(theta)
    g = prop.gradient()
    assert J > 0 and np.abs(g).max() > 0
    step = 1e-5
    fd = np.array([(prop.forward(theta + step * e, keep=False) - prop.forward(theta - step * e, keep=False)) / (2 * step)
                   for e in np.eye(len(theta))])
    assert np.abs(g - fd).max() <= 1e-6 * np.abs(g).max(), (g, fd)
    Phi = P.Phi.cpu().numpy()
    outer = P.outer.cpu().numpy().real
    tables = cpu.host_tables(h)

    def objective(th):
        E = prop.fields(th)
        x = psi0.copy()
        for n in range(prop.steps):
            x, _ = arnoldi.exponential_action(
                lambda y, e=E[n]: cpu.tensor_apply(h, y, (0., 0., e), False, tables=tables), x, prop.dt, 1e-13, 30)
        u = x.reshape((h.n, h.n, h.nc), order='F')
        a = np.einsum('ci,ijc->jc', Phi.conj(), u)
        return float(np.sum(outer[:, None] * np.abs(a) ** 2))

    with threadpool_limits(limits=1, user_api='blas'):
        assert abs(objective(theta) - J) <= 1e-10 * J
        ref = np.array([(objective(theta + step * e) - objective(theta - step * e)) / (2 * step)
                        for e in np.eye(len(theta))])
    assert np.abs(g - ref).max() <= 1e-6 * np.abs(ref).max(), (g, ref)
