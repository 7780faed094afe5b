"""GPU parity on bipolar all-M channel tables (production circular / pump-probe inputs):
H·psi with a field that has x, y and z components (complex Cartesian dipole coefficients)
against the reference's own outputs on the same tables (Kronecker assembly of the product
basis projected by the bipolar isometry, and TorchHamiltonian), every kernel path, complex64,
batched instances, the surface flux and an Arnoldi step against the oracle.

Tolerances: complex128 at the reference's kernel-vs-Kronecker bound (rtol 2e-13,
atol 2e-12); complex64 within 2e-6 relative L2; Arnoldi within 1e-12 relative L2."""
import numpy as np
import pytest
import torch

from oracle import arnoldi, cpu
from test_bipolar import build

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'


def engine(h):
    from laqphysics_b200.engine import B200Hamiltonian
    return B200Hamiltonian(h, DEVICE)


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize('gauge', ['length', 'velocity'])
def test_bipolar_apply_matches_reference_every_path(gauge):
    g, b = build()
    op = engine(b)
    assert op.tiled and op.plan_info['band_kernel']
    x = op.state(g['x'])
    velocity = gauge == 'velocity'
    for path in (1, 3, 2, 0):
        op.set_path(path)
        y = op.host(op.apply(x, g['field'], velocity))
        np.testing.assert_allclose(y, g[f'kron_{gauge}'], rtol=2e-13, atol=2e-12, err_msg=str(path))
        np.testing.assert_allclose(y, g[f'torch_{gauge}'], rtol=2e-13, atol=2e-12, err_msg=str(path))
        y64 = op.host(op.apply(x.to(torch.complex64), g['field'], velocity, precision='complex64'))
        assert rel_l2(y64.astype(complex), g[f'kron_{gauge}']) < 2e-6, path
    op.set_path(1)
    op.synchronize()


def test_bipolar_batched_circular_fields():
    g, b = build()
    op = engine(b)
    rng = np.random.default_rng(5)
    count = 4
    fields = rng.uniform(-.05, .05, (count, 3))
    x = torch.stack([op.state(g['x']) * (k + 1) for k in range(count)]).contiguous()
    for velocity in (False, True):
        y = op.apply_batched(x, fields, velocity)
        for k in range(count):
            ref = cpu.tensor_apply(b, op.host(x[k]), fields[k], velocity)
            assert rel_l2(op.host(y[k]), ref) < 1e-13
    op.synchronize()


def test_bipolar_surface_flux_and_arnoldi_step():
    from laqphysics_b200.torch_backend import FieldOperator, exponential_action
    g, b = build()
    b.prepare_surface(5)
    op = engine(b)
    x = g['x'] / np.linalg.norm(g['x'])
    f = np.array([.02, -.01, .015])
    np.testing.assert_allclose(op.flux(op.state(x), f), b.flux(x, f), rtol=2e-12, atol=2e-12)
    y, info = exponential_action(FieldOperator(op, f, False), op.state(x), .01, tol=1e-11, maxdim=24)
    ref, rinfo = arnoldi.exponential_action(lambda v: cpu.tensor_apply(b, v, f, False), x, .01, tol=1e-11, maxdim=24)
    assert info['dimension'] == rinfo['dimension']
    assert rel_l2(op.host(y), ref) < 1e-12


def test_bipolar_surface_contraction_matches_reference():
    """Ionic contraction of a surface frame in the bipolar all-M basis (unfolded He+ labels
    with m = -1, 0, 1) against the reference's sparse-transform contraction, 1e-12."""
    import json as js
    from scipy.sparse import csr_matrix
    from conftest import golden
    from laqphysics_b200.bipolar import BipolarHelium
    from laqphysics_b200.fedvr import make_grid
    from laqphysics_b200.surface3d import Ionic
    from laqphysics_b200.surface_contract import SurfaceContractor
    g = golden('bipolar_contraction')
    h = BipolarHelium(make_grid(**js.loads(str(g['grid']))), lmax=1, total_Lmax=1, M=None,
                      cutoff_radii=tuple(g['cutoff']))
    base = h.uncoupled
    base.prepare_surface(float(g['surface']))
    ion = Ionic(base, None)
    labels = [tuple(int(v) for v in x) for x in g['labels']]
    for transform in (h.transform, csr_matrix(h.transform)):
        contract = SurfaceContractor(base, ion, labels, labels, list(range(len(labels))), False, transform, DEVICE)
        assert contract.outerstates == [tuple(int(v) for v in x) for x in g['outer']]
        q = contract(g['chi'], g['frame'])
        np.testing.assert_allclose(q, g['q'], rtol=1e-12, atol=1e-12)
