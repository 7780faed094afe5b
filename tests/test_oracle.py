"""Pin the CPU oracle to the reference's own outputs (golden fixtures).

The C restatement of src/kernels.f90:119-176 must reproduce the reference's
independent Kronecker assembly (python/helium3d.py:105-123) and its PyTorch backend
at the reference's own tolerance (tests/test_kernels.py:31-37: rtol 2e-13,
atol 2e-12); the numpy Arnoldi must reproduce python/propagate.py.
"""
import numpy as np
import pytest

from conftest import Tables, golden
from oracle import arnoldi, cpu

CASES = ['apply_ecs', 'apply_cut', 'apply_coupled']


@pytest.mark.parametrize('case', CASES)
@pytest.mark.parametrize('gauge', ['length', 'velocity'])
def test_oracle_matches_reference_kronecker_and_torch(case, gauge):
    g = golden(case)
    h = Tables(g)
    out = cpu.tensor_apply(h, g['x'], g['field'], gauge == 'velocity')
    np.testing.assert_allclose(out, g[f'kron_{gauge}'], rtol=2e-13, atol=2e-12)
    np.testing.assert_allclose(out, g[f'torch_{gauge}'], rtol=2e-13, atol=2e-12)


def test_oracle_zero_field_skips_dipoles_and_a2():
    g = golden('apply_cut')
    h = Tables(g)
    x = g['x']
    length = cpu.tensor_apply(h, x, (0., 0., 0.), False)
    velocity = cpu.tensor_apply(h, x, (0., 0., 0.), True)
    np.testing.assert_array_equal(length, velocity)


def test_oracle_arnoldi_matches_reference_dense_case():
    g = golden('arnoldi_dense')
    y, info = arnoldi.exponential_action(lambda z: g['H'] @ z, g['x'], float(g['dt']), tol=float(g['tol']))
    assert info['dimension'] == int(g['dimension'])
    np.testing.assert_allclose(y, g['y'], atol=1e-13, rtol=1e-13)
    np.testing.assert_allclose(y, g['exact'], atol=2e-11, rtol=2e-11)


def test_oracle_arnoldi_matches_reference_on_helium_operator():
    g = golden('apply_cut')
    h = Tables(g)
    f = g['field']
    y, info = arnoldi.exponential_action(lambda v: cpu.tensor_apply(h, v, f, True), g['x'], float(g['arnoldi_dt']),
                                         tol=float(g['arnoldi_tol']))
    assert info['dimension'] == int(g['arnoldi_cpu_dim'])
    np.testing.assert_allclose(y, g['arnoldi_cpu'], atol=2e-12, rtol=2e-12)
    np.testing.assert_allclose(y, g['arnoldi_torch'], atol=2e-11, rtol=2e-11)


def test_oracle_step_halves_dt_when_krylov_space_too_small():
    g = golden('arnoldi_dense')
    H = g['H']
    with pytest.raises(RuntimeError, match='Arnoldi did not converge'):
        arnoldi.exponential_action(lambda z: H @ z, g['x'], 1.0, tol=1e-10, maxdim=8)
    y, info = arnoldi.step(lambda t, z: H @ z, g['x'], 0., 1.0, tol=1e-10, maxdim=8)
    from scipy.linalg import expm
    np.testing.assert_allclose(y, expm(-1j * H) @ g['x'], atol=1e-9, rtol=1e-9)
    assert info.get('subdivided')
