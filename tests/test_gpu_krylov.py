"""GPU parity of the Arnoldi exponential (device CGS2, on-device expm, device checks)
against the reference's own results (golden fixtures from python/propagate.py and
python/torch_backend.py) and the numpy oracle.  Tolerance: the reference's own
Torch-vs-Fortran Arnoldi bound (tests/test_torch_backend.py:18-20: 2e-11)."""
import json

import numpy as np
import pytest
import torch

from conftest import Tables, golden
from oracle import arnoldi, cpu

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'


def engine(h):
    from laqphysics_b200.engine import B200Hamiltonian
    return B200Hamiltonian(h, DEVICE)


@pytest.mark.parametrize('fused', [False, True])
def test_arnoldi_matches_reference_on_helium(fused):
    from laqphysics_b200.torch_backend import FieldOperator, exponential_action
    g = golden('apply_cut')
    op = engine(Tables(g))
    f = g['field']
    apply = FieldOperator(op, f, True) if fused else (lambda y: op.apply(y, f))
    y, info = exponential_action(apply, op.state(g['x']), float(g['arnoldi_dt']), tol=float(g['arnoldi_tol']))
    assert info['dimension'] == int(g['arnoldi_torch_dim'])
    np.testing.assert_allclose(op.host(y), g['arnoldi_torch'], atol=2e-11, rtol=2e-11)
    np.testing.assert_allclose(op.host(y), g['arnoldi_cpu'], atol=2e-11, rtol=2e-11)


def test_arnoldi_dense_reference_case():
    from laqphysics_b200.torch_backend import exponential_action
    g = golden('arnoldi_dense')
    H = torch.tensor(g['H'], device=DEVICE)
    y, info = exponential_action(lambda z: H @ z, torch.tensor(g['x'], device=DEVICE), float(g['dt']),
                                 tol=float(g['tol']), maxdim=60)
    assert info['dimension'] == int(g['dimension'])
    np.testing.assert_allclose(y.cpu().numpy(), g['y'], atol=1e-12, rtol=1e-12)
    np.testing.assert_allclose(y.cpu().numpy(), g['exact'], atol=2e-11, rtol=2e-11)


def test_arnoldi_reports_non_convergence_with_reference_message():
    from laqphysics_b200.torch_backend import exponential_action
    g = golden('arnoldi_dense')
    H = torch.tensor(g['H'], device=DEVICE)
    with pytest.raises(RuntimeError, match='Arnoldi did not converge'):
        exponential_action(lambda z: H @ z, torch.tensor(g['x'], device=DEVICE), 1.0, tol=1e-10, maxdim=8)


def test_step_subdivides_like_the_oracle():
    from laqphysics_b200.torch_backend import step
    g = golden('arnoldi_dense')
    H = torch.tensor(g['H'], device=DEVICE)
    y, info = step(lambda t, z: H @ z, torch.tensor(g['x'], device=DEVICE), 0., 1.0, tol=1e-10, maxdim=8)
    ref, rinfo = arnoldi.step(lambda t, z: g['H'] @ z, g['x'], 0., 1.0, tol=1e-10, maxdim=8)
    assert info.get('subdivided') and rinfo.get('subdivided')
    np.testing.assert_allclose(y.cpu().numpy(), ref, atol=1e-11, rtol=1e-11)


def _length_run_setup():
    from laqphysics_b200.pulses import Pulse
    from laqphysics_b200.workloads import coupled
    g = golden('length_run')
    grid = json.loads(str(g['grid']))
    h = coupled(grid['edges'], grid['order'], int(g['lmax']), int(g['total_Lmax']), ecs_angle=grid['ecs_angle'],
                tail=grid['tail'], cutoff_radii=tuple(g['cutoff']))
    return g, h, Pulse(**json.loads(str(g['pulse'])))


@pytest.mark.parametrize('fused', [False, True])
def test_length_gauge_propagation_matches_reference(fused):
    """Six midpoint Arnoldi steps in the length gauge (python/propagate.py:41-50 driven like
    python/run3d.py:196-199) agree with the reference's complex128 run to 1e-10 rel L2."""
    from laqphysics_b200.torch_backend import FieldSchedule, step
    g, h, pulse = _length_run_setup()
    op = engine(h)
    field = lambda t: (0., 0., float(pulse.electric(t)))
    apply_at = FieldSchedule(op, field, False) if fused else (lambda t, v: op.apply(v, field(t), False))
    y = op.state(g['states'][0])
    dt = float(g['dt'])
    for i in range(len(g['dimensions'])):
        y, info = step(apply_at, y, i * dt, dt, tol=float(g['tol']), maxdim=int(g['maxdim']))
        assert info['dimension'] == int(g['dimensions'][i])
        ref = g['states'][i + 1]
        assert np.linalg.norm(op.host(y) - ref) / np.linalg.norm(ref) < 1e-10


def test_mixed_precision_propagation_against_fp64_reference():
    """complex64 H·psi inside the complex128 Krylov process: the six-step length-gauge run
    stays within 1e-5 relative L2 of the reference's complex128 states (stated mixed
    tolerance), conserves the norm to 1e-6 and keeps the reference's Krylov dimensions;
    the generic callable path agrees with the fused one to 1e-6."""
    from laqphysics_b200.torch_backend import FieldSchedule, step
    g, h, pulse = _length_run_setup()
    from laqphysics_b200.engine import B200Hamiltonian
    op = B200Hamiltonian(h, DEVICE)
    field = lambda t: (0., 0., float(pulse.electric(t)))
    fused = FieldSchedule(op, field, False, precision='mixed')
    generic = lambda t, v: fused.at(t)(v)
    y = op.state(g['states'][0])
    z = op.state(g['states'][0])
    dt = float(g['dt'])
    for i in range(len(g['dimensions'])):
        y, info = step(fused, y, i * dt, dt, tol=float(g['tol']), maxdim=int(g['maxdim']))
        z, _ = step(generic, z, i * dt, dt, tol=float(g['tol']), maxdim=int(g['maxdim']))
        assert info['dimension'] == int(g['dimensions'][i])
        ref = g['states'][i + 1]
        assert np.linalg.norm(op.host(y) - ref) / np.linalg.norm(ref) < 1e-5
        assert abs(np.linalg.norm(op.host(y)) - np.linalg.norm(ref)) < 1e-6
    assert np.linalg.norm(op.host(y) - op.host(z)) / np.linalg.norm(op.host(z)) < 1e-6


def test_fused_and_generic_arnoldi_agree_on_larger_grid():
    from laqphysics_b200.torch_backend import FieldOperator, exponential_action
    from laqphysics_b200.workloads import coupled, seeded_state
    h = coupled(np.linspace(0, 30, 16), 8, 3, 2, ecs_angle=.3, tail=12, cutoff_radii=(20., 25.))
    op = engine(h)
    x = op.state(seeded_state(h.size, 21))
    f = (0., 0., .03)
    a, ia = exponential_action(FieldOperator(op, f, False), x, .005, tol=1e-10, maxdim=16)
    b, ib = exponential_action(lambda y: op.apply(y, f, False), x, .005, tol=1e-10, maxdim=16)
    c, ic = arnoldi.exponential_action(lambda v: cpu.tensor_apply(h, v, f, False), op.host(x), .005, tol=1e-10,
                                       maxdim=16)
    assert ia['dimension'] == ib['dimension'] == ic['dimension']
    # the fused loop takes h_{j+1,j} from the second CGS sweep (|v'|^2 - |z'|^2), the host
    # loop from a separate norm: equal up to rounding
    assert np.linalg.norm(op.host(a) - op.host(b)) / np.linalg.norm(op.host(b)) < 1e-13
    assert np.linalg.norm(op.host(a) - c) / np.linalg.norm(c) < 1e-12


@pytest.mark.parametrize('precision', ['complex128', 'mixed'])
def test_batched_arnoldi_matches_single_instance_steps(precision):
    """he_expv_batched (every instance of the batch in one launch per kernel) against the
    same instances stepped one by one: the per-instance arithmetic is the same, so the
    states agree to rounding."""
    from laqphysics_b200.torch_backend import FieldSchedule, step, step_batched
    from laqphysics_b200.workloads import arnoldi_small, seeded_state
    h = arnoldi_small()
    op = engine(h)
    count = 4
    peaks = np.array([.005, .01, .02, .03])
    fields_at = lambda t: np.stack([[0., 0., p * np.sin(1.6 * t)] for p in peaks])
    x0 = torch.stack([op.state(seeded_state(h.size, 50 + b)) for b in range(count)])
    x0 /= torch.linalg.vector_norm(x0, dim=1, keepdim=True)
    dt, tol, maxdim = .01, 1e-10, 12
    xb = x0.clone()
    for i in range(3):
        xb, info = step_batched(op, fields_at, xb, i * dt, dt, tol, maxdim, precision=precision)
    for b in range(count):
        schedule = FieldSchedule(op, lambda t, b=b: fields_at(t)[b], velocity=False, precision=precision)
        xs = x0[b].contiguous()
        for i in range(3):
            xs, _ = step(schedule, xs, i * dt, dt, tol, maxdim)
        err = float(torch.linalg.vector_norm(xb[b] - xs) / torch.linalg.vector_norm(xs))
        assert err < 1e-13, (b, err)
    assert (info['dimension'] <= maxdim).all()


@pytest.mark.parametrize('precision', ['complex128', 'mixed'])
def test_graph_replayed_arnoldi_steps_match_direct_launches(precision):
    """Repeated solves replayed as one captured CUDA graph (new state, field and dt each
    time) give bit-identical results to the directly launched solves, single and batched."""
    from laqphysics_b200 import torch_backend as tb
    from laqphysics_b200.torch_backend import FieldSchedule, step, step_batched
    from laqphysics_b200.workloads import arnoldi_small, seeded_state
    h = arnoldi_small()
    op = engine(h)
    x0 = op.state(seeded_state(h.size, 5))
    x0 /= torch.linalg.vector_norm(x0)
    field = lambda t: (0., 0., .01 * np.sin(t + .3))
    fields = lambda t: np.array([[0., 0., .01 * np.sin(t + .3 * b)] for b in range(3)])
    runs = {}
    previous = tb.use_cuda_graphs(True)
    for graphs in (False, True):
        tb.use_cuda_graphs(graphs)
        try:
            sched = FieldSchedule(op, field, velocity=False, precision=precision)
            x, xb = x0.clone(), x0.repeat(3).reshape(3, -1).contiguous()
            for i in range(4):
                x, _ = step(sched, x, i * .005, .005, 1e-10, 16)
                xb, _ = step_batched(op, fields, xb, i * .005, .005, 1e-10, 16, precision=precision)
            runs[graphs] = (op.host(x), xb.cpu().numpy())
        finally:
            tb.use_cuda_graphs(previous)
    np.testing.assert_array_equal(runs[True][0], runs[False][0])
    np.testing.assert_array_equal(runs[True][1], runs[False][1])
    op.synchronize()


@pytest.mark.parametrize('precision', ['complex128', 'mixed'])
def test_applies_past_convergence_do_no_work(precision):
    """A fused solve enqueues all maxdim iterations; the H·psi launches after its device-side
    convergence return without work.  The result and dimension do not depend on maxdim, and
    the extra iterations cost far less than applies (timed with CUDA events)."""
    from laqphysics_b200.torch_backend import FieldOperator, exponential_action
    from laqphysics_b200.workloads import arnoldi_small, seeded_state
    h = arnoldi_small()
    op = engine(h)
    x = op.state(seeded_state(h.size, 9))
    x /= torch.linalg.vector_norm(x)
    apply = FieldOperator(op, (0., 0., .01), velocity=False, precision=precision)
    loose, info = exponential_action(apply, x, .002, 1e-8, 48)
    small = info['dimension'] + 1
    assert small < 40
    tight, info2 = exponential_action(apply, x, .002, 1e-8, small)
    assert info['dimension'] == info2['dimension']
    np.testing.assert_allclose(op.host(loose), op.host(tight), rtol=1e-14, atol=1e-16)

    def timed(run, reps=5):
        run()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(reps):
            run()
        stop.record()
        torch.cuda.synchronize()
        return start.elapsed_time(stop) / reps

    t_small = timed(lambda: exponential_action(apply, x, .002, 1e-8, small))
    t48 = timed(lambda: exponential_action(apply, x, .002, 1e-8, 48))
    t_apply = timed(lambda: apply(x), reps=20)
    # each extra iteration is a handful of empty launches, not an apply
    assert (t48 - t_small) / (48 - small) < 0.6 * t_apply, (t_small, t48, t_apply)


def test_graph_capture_fallback_counter_starts_at_zero():
    """Repeated solves replay as graphs without a capture fallback in a single thread."""
    import ctypes as ct
    from laqphysics_b200._lib import LIB
    from laqphysics_b200.torch_backend import FieldOperator, exponential_action, workspace
    from laqphysics_b200.workloads import coupled, seeded_state
    h = coupled(np.linspace(0, 12, 7), 5, 2, 2, ecs_angle=.3, tail=8, cutoff_radii=(1., 1.8))
    op = engine(h)
    x = op.state(seeded_state(h.size, 4))
    for _ in range(4):
        exponential_action(FieldOperator(op, (0., 0., .05), False), x, .005, 1e-11, 16)
    ws = workspace(h.size, 16, op.device)
    fallbacks, graphs = ct.c_int(-1), ct.c_int(-1)
    assert LIB.he_krylov_capture_fallbacks(ws.handle, ct.byref(fallbacks), ct.byref(graphs)) == 0
    assert fallbacks.value == 0 and graphs.value == 1
