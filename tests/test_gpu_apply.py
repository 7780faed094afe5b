"""GPU parity of H·psi: the sm_100a kernels against the reference's own outputs
(golden fixtures) and against the CPU oracle at sizes beyond the fixtures.

Tolerances: complex128 uses the reference's own kernel-vs-Kronecker bound
(tests/test_kernels.py:37: rtol 2e-13, atol 2e-12); complex64 is held to a relative
L2 error of 2e-6 against the complex128 oracle.
"""
import json

import numpy as np
import pytest
import torch

from conftest import Tables, golden
from oracle import cpu

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'
C64_REL_L2 = 2e-6


def engine(h, **kw):
    from laqphysics_b200.engine import B200Hamiltonian
    return B200Hamiltonian(h, DEVICE, **kw)


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize('case', ['apply_ecs', 'apply_cut', 'apply_coupled'])
@pytest.mark.parametrize('gauge', ['length', 'velocity'])
def test_apply_matches_reference_goldens(case, gauge):
    g = golden(case)
    op = engine(Tables(g))
    y = op.host(op.apply(op.state(g['x']), g['field'], gauge == 'velocity'))
    np.testing.assert_allclose(y, g[f'kron_{gauge}'], rtol=2e-13, atol=2e-12)
    np.testing.assert_allclose(y, g[f'torch_{gauge}'], rtol=2e-13, atol=2e-12)


def _coupled(edges, order, angle, tail, lmax, L, cut=(2., 3.)):
    from laqphysics_b200.coupled_angular import CoupledHelium
    from laqphysics_b200.fedvr import make_grid
    from laqphysics_b200.helium3d import Helium
    return CoupledHelium(Helium(make_grid(edges, order, ecs_angle=angle, tail=tail), lmax, M=0, cutoff_radii=cut), L)


def test_separable_diagonal_path_matches_reference_goldens():
    g = golden('apply_coupled')
    h = _coupled(**dict(zip(('edges', 'order', 'angle', 'tail'), json.loads(str(g['grid'])).values())), lmax=2, L=2,
                 cut=(1., 2.))
    assert hasattr(h, 'diag_parts')
    op = engine(h)
    for gauge in ('length', 'velocity'):
        y = op.host(op.apply(op.state(g['x']), g['field'], gauge == 'velocity'))
        np.testing.assert_allclose(y, g[f'kron_{gauge}'], rtol=2e-13, atol=2e-12)


@pytest.mark.parametrize('velocity', [False, True])
def test_apply_matches_oracle_on_larger_coupled_grid(velocity):
    h = _coupled(np.linspace(0, 30, 16), 8, .3, 12, 3, 2)
    rng = np.random.default_rng(7)
    x = rng.normal(size=h.size) + 1j * rng.normal(size=h.size)
    f = (0., 0., .07)
    op = engine(h)
    y = op.host(op.apply(op.state(x), f, velocity))
    ref = cpu.tensor_apply(h, x, f, velocity)
    assert rel_l2(y, ref) < 1e-13
    np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize('velocity', [False, True])
def test_tiled_and_generic_kernels_agree(velocity):
    h = _coupled(np.linspace(0, 30, 16), 8, .3, 12, 3, 2)
    op = engine(h)
    assert op.tiled
    rng = np.random.default_rng(17)
    x = op.state(rng.normal(size=h.size) + 1j * rng.normal(size=h.size))
    f = (0., 0., .2)
    a = op.host(op.apply(x, f, velocity))
    op.use_tiled(False)
    b = op.host(op.apply(x, f, velocity))
    op.use_tiled(True)
    assert rel_l2(a, b) < 1e-14
    alpha = .05 / (3 - 1j * np.sqrt(3))
    c = op.host(op.apply_shifted(x, f, alpha, -2.9, velocity=velocity))
    np.testing.assert_allclose(c, op.host(x) + 1j * alpha * (b + 2.9 * op.host(x)), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize('velocity', [False, True])
def test_kinetic_tma_and_shared_memory_radial_kernels_agree(velocity):
    """Path 1 (banded FP64 tensor-core kinetic kernel for complex128, TMA-staged FMA
    kinetic kernel for complex64), path 3 (TMA-staged FMA kinetic kernel), path 2
    (shared-memory radial kernel) and path 0 (generic kernel) in both precisions, on a
    grid whose exterior tail is split over column slots and whose last row group is
    ragged."""
    h = _coupled(np.linspace(0, 24, 7), 6, .3, 24, 2, 1, cut=(12., 15.))
    op = engine(h)
    rng = np.random.default_rng(23)
    x = op.state(rng.normal(size=h.size) + 1j * rng.normal(size=h.size))
    f = (0., 0., .15)
    results = {}
    for path in (1, 3, 2, 0):
        op.set_path(path)
        results[path] = (op.host(op.apply(x, f, velocity)),
                         op.host(op.apply(x.to(torch.complex64), f, velocity, precision='complex64')))
    op.set_path(1)
    op.synchronize()
    ref = cpu.tensor_apply(h, op.host(x), f, velocity)
    for path, (y, y64) in results.items():
        assert rel_l2(y, ref) < 1e-13, path
        assert rel_l2(y64.astype(complex), ref) < C64_REL_L2, path


def test_microbenchmark_grid_apply_matches_oracle():
    from laqphysics_b200.workloads import hpsi_microbench, seeded_state
    h = hpsi_microbench()
    op = engine(h)
    assert op.tiled
    x = seeded_state(h.size, 1234)
    for velocity in (False, True):
        y = op.host(op.apply(op.state(x), (0., 0., .02), velocity))
        ref = cpu.tensor_apply(h, x, (0., 0., .02), velocity)
        assert rel_l2(y, ref) < 1e-13
        y64 = op.host(op.apply(op.state(x).to(torch.complex64), (0., 0., .02), velocity, precision='complex64'))
        assert rel_l2(y64.astype(complex), ref) < C64_REL_L2


def test_complex64_apply_within_stated_tolerance():
    h = _coupled(np.linspace(0, 30, 16), 8, .3, 12, 3, 2)
    rng = np.random.default_rng(8)
    x = rng.normal(size=h.size) + 1j * rng.normal(size=h.size)
    x /= np.linalg.norm(x)
    op = engine(h)
    ref = cpu.tensor_apply(h, x, (0, 0, .05), False)
    y = op.apply(op.state(x).to(torch.complex64), (0, 0, .05), False, precision='complex64')
    assert y.dtype == torch.complex64
    assert rel_l2(op.host(y).astype(complex), ref) < C64_REL_L2


def test_shifted_pade_operator():
    g = golden('apply_cut')
    h = Tables(g)
    op = engine(h)
    alpha = .05 / (3 + 1j * np.sqrt(3))
    x = g['x']
    y = op.host(op.apply_shifted(op.state(x), g['field'], alpha, -2.9, velocity=True))
    ref = x + 1j * alpha * (cpu.tensor_apply(h, x, g['field'], True) + 2.9 * x)
    np.testing.assert_allclose(y, ref, rtol=1e-13, atol=1e-13)


def test_jacobi_diagonal_matches_reference_formula():
    g = golden('apply_cut')
    h = Tables(g)
    op = engine(h)
    n, nc = h.n, h.nc
    td = np.array([h.tv[k] for i in range(n) for k in range(h.ptr[i], h.ptr[i + 1]) if h.col[k] == i])
    d = h.diag.copy()
    d += td[:, None, None] + td[None, :, None]
    for a in range(nc):
        for k in range(h.vptr[a], h.vptr[a + 1]):
            if h.vc[k] == a:
                d[:, :, a] += h.vcoef[k] * h.rad[:, :, h.vl[k]]
    np.testing.assert_allclose(op.host(op.diagonal), d.ravel(order='F'), rtol=1e-14, atol=1e-13)


def test_flux_matches_reference():
    g = golden('apply_cut')
    h = Tables(g)
    h.surface_indices, h.surface_T, h.surface_P = g['surface_indices'], g['surface_T'], g['surface_P']
    op = engine(h)
    frame = op.flux(op.state(g['x']), g['field'])
    np.testing.assert_allclose(frame, g['flux'], rtol=2e-12, atol=2e-12)
    np.testing.assert_allclose(frame, g['flux_torch'], rtol=2e-12, atol=2e-12)


def test_coupled_flux_matches_reference():
    g = golden('apply_coupled')
    args = json.loads(str(g['grid']))
    h = _coupled(args['edges'], args['order'], args['ecs_angle'], args['tail'], 2, 2, cut=(1., 2.))
    h.prepare_surface(5)
    op = engine(h)
    np.testing.assert_allclose(op.flux(op.state(g['x']), g['field']), g['flux'], rtol=2e-12, atol=2e-12)


def test_host_pointer_tensor_apply_drop_in():
    from laqphysics_b200.native import tensor_apply
    g = golden('apply_ecs')
    h = Tables(g)
    for gauge in ('length', 'velocity'):
        y = tensor_apply(h, g['x'], g['field'], gauge == 'velocity')
        np.testing.assert_allclose(y, g[f'kron_{gauge}'], rtol=2e-13, atol=2e-12)


def test_apply_rejects_wrong_dtype_and_size():
    op = engine(Tables(golden('apply_ecs')))
    with pytest.raises(ValueError):
        op.apply(torch.zeros(op.size, dtype=torch.complex64, device=DEVICE), precision='complex128')
    with pytest.raises(ValueError):
        op.apply(torch.zeros(op.size + 1, dtype=torch.complex128, device=DEVICE))


@pytest.mark.parametrize('velocity', [False, True])
def test_batched_apply_matches_single_applies(velocity):
    """he_apply_batched (one launch per kernel for the whole batch) against one apply per
    instance, complex128 and complex64, instances with different fields."""
    from laqphysics_b200.workloads import arnoldi_small, seeded_state
    h = arnoldi_small()
    op = engine(h)
    count = 5
    rng = np.random.default_rng(31)
    fields = np.zeros((count, 3))
    fields[:, 2] = rng.uniform(.005, .03, count)
    x = torch.stack([op.state(seeded_state(h.size, 100 + b)) for b in range(count)])
    for dtype, precision, tol in ((torch.complex128, 'complex128', 1e-14), (torch.complex64, 'complex64', 1e-6)):
        xb = x.to(dtype).contiguous()
        y = op.apply_batched(xb, fields, velocity, precision=precision)
        for b in range(count):
            yb = op.apply(xb[b].contiguous(), fields[b], velocity, precision=precision)
            assert rel_l2(op.host(y[b]).astype(complex), op.host(yb).astype(complex)) < tol, (precision, b)
        ref = cpu.tensor_apply(h, op.host(x[count - 1]), fields[count - 1], velocity)
        assert rel_l2(op.host(y[count - 1]).astype(complex), ref) < (1e-13 if precision == 'complex128' else C64_REL_L2)
    op.synchronize()


def test_fp64_peak_probes():
    from laqphysics_b200.engine import fp64_peaks
    p = fp64_peaks(DEVICE, iters=256)
    assert p['dmma'] > 1.0 and p['dfma'] > 1.0


def test_mixing_kernel_occupancy_choices_agree():
    """The autotuner's candidates (register budgets of the generated mixing kernel) give
    the same H·psi; the fastest one stays selected."""
    from laqphysics_b200.workloads import arnoldi_small, seeded_state
    h = arnoldi_small()
    op = engine(h)
    x = op.state(seeded_state(h.size, 41))
    f = (0., 0., .02)
    ref = op.host(op.apply(x, f, False))
    timings = op.autotune(f, False, precisions=('complex128',), candidates=(2, 4), reps=2)
    assert set(timings['complex128']['mix_blocks']) == {2, 4} and set(timings['complex128']['band_stages']) == {1, 2}
    for blocks in (2, 4):
        op.set_mix_blocks('complex128', blocks)
        np.testing.assert_array_equal(op.host(op.apply(x, f, False)), ref)
    op.synchronize()


@pytest.mark.parametrize('precision', ['complex128', 'complex64'])
def test_band_kernel_single_and_double_stage_forms_agree(precision):
    """The one-stage, two-CTA form of the banded kinetic kernel gives bit-identical H·psi to
    the two-stage form, on a grid with a ragged last tile and on a batch of instances."""
    from laqphysics_b200.workloads import arnoldi_small, seeded_state
    h = _coupled(np.linspace(0, 24, 7), 6, .3, 24, 2, 1, cut=(12., 15.))
    dtype = torch.complex128 if precision == 'complex128' else torch.complex64
    for hh in (h, arnoldi_small()):
        op = engine(hh)
        x = op.state(seeded_state(hh.size, 43)).to(dtype)
        f = (0., 0., .03)
        fields = np.array([[0., 0., .01], [0., 0., .02], [0., 0., .03]])
        xb = torch.stack([x, 2 * x, -x]).contiguous()
        results = {}
        for stages in (2, 1):
            op.set_band_stages(precision, stages)
            results[stages] = (op.host(op.apply(x, f, False, precision=precision)),
                               op.host(op.apply_batched(xb, fields, False, precision=precision)))
        op.synchronize()
        np.testing.assert_array_equal(results[1][0], results[2][0])
        np.testing.assert_array_equal(results[1][1], results[2][1])


def test_host_stream_apply_matches_device_apply():
    """apply_host_stream (H2D, apply and D2H of consecutive host states overlapped on three
    streams) returns exactly the per-state device results, for more states than buffers."""
    from laqphysics_b200.workloads import arnoldi_small, seeded_state
    h = arnoldi_small()
    op = engine(h)
    xs = [torch.as_tensor(seeded_state(h.size, 60 + k)).pin_memory() for k in range(5)]
    f = (0., 0., .02)
    outs = op.apply_host_stream(xs, f, False)
    for x, y in zip(xs, outs):
        ref = op.host(op.apply(x.to(DEVICE), f, False))
        np.testing.assert_array_equal(y.numpy(), ref)
    outs64 = op.apply_host_stream([x.to(torch.complex64).pin_memory() for x in xs], f, True, precision='complex64')
    ref = op.host(op.apply(xs[3].to(DEVICE).to(torch.complex64), f, True, precision='complex64'))
    np.testing.assert_array_equal(outs64[3].numpy(), ref)
    op.synchronize()


def test_kernels_run_as_sm100a_binaries():
    """cudaFuncGetAttributes(binaryVersion) of a library kernel as loaded on the B200."""
    import ctypes as ct
    from laqphysics_b200._lib import LIB
    torch.zeros(1, device=DEVICE)
    version = ct.c_int()
    assert LIB.he_binary_version(ct.byref(version)) == 0, LIB.he_last_error().decode()
    assert version.value == 100


@pytest.mark.parametrize('basis', ['coupled', 'product'])
def test_device_run_diagnostics_match_the_driver_formulas(basis):
    """B200Hamiltonian.diagnostics (he_diagnostics) against python/run3d.py:212-224's host
    formulas on the host copy: real-region norm with the interior mass fraction, ground
    population |<g|psi>|^2 and the exchange error (coupled: with the (-1)^(l1+l2-L) sign)."""
    from laqphysics_b200.fedvr import make_grid
    from laqphysics_b200.helium3d import Helium
    from laqphysics_b200.workloads import coupled, seeded_state
    if basis == 'coupled':
        h = coupled(np.linspace(0, 12, 7), 5, 2, 2, ecs_angle=.3, tail=8, cutoff_radii=(1., 1.8))
    else:
        h = Helium(make_grid(np.linspace(0, 12, 7), 5, ecs_angle=.3, tail=8), 1, M=None, cutoff_radii=(1., 1.8))
    op = engine(h)
    x, gs = seeded_state(h.size, 5), seeded_state(h.size, 6)
    d = op.diagnostics(op.state(x), op.state(gs))
    u = x.reshape(h.shape, order='F')
    f = h.grid.interior_weights / abs(h.grid.weights)
    norm = float(np.sum(abs(u) ** 2 * f[:, None, None] * f[None, :, None]))
    assert abs(d['real_region_norm'] - norm) <= 1e-13 * norm
    assert abs(d['ground_population'] - abs(np.vdot(gs, x)) ** 2) <= 1e-13
    assert abs(d['exchange_error'] - h.exchange_error(x)) <= 1e-12 * h.exchange_error(x)
