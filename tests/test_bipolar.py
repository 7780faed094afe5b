"""Bipolar all-M channel tables (laqphysics_b200.bipolar) against the reference's own
BipolarHelium tables (tests/golden/apply_bipolar.npz, made by tests/golden/make_golden.py):
same basis and edge structure exactly, coefficients within 1e-13."""
import json

import numpy as np

from conftest import golden


def build(M=None, natural_parity=False, lmax=2, total_Lmax=2):
    from laqphysics_b200.bipolar import BipolarHelium
    from laqphysics_b200.fedvr import make_grid
    g = golden('apply_bipolar')
    return g, BipolarHelium(make_grid(**json.loads(str(g['grid']))), lmax=lmax, total_Lmax=total_Lmax, M=M,
                            cutoff_radii=tuple(g['cutoff']), natural_parity=natural_parity)


def test_bipolar_tables_match_reference():
    g, b = build()
    assert b.shape == tuple(g['shape'])
    np.testing.assert_array_equal(np.array(b.basis), g['basis'])
    for name in ('vptr', 'vc', 'vl', 'dptr', 'dc', 'de', 'exchange', 'ptr', 'col'):
        np.testing.assert_array_equal(getattr(b, name), g['t_' + name], err_msg=name)
    for name in ('vcoef', 'dcoef', 'ldiff', 'rad', 'diag', 'tv', 'r'):
        np.testing.assert_allclose(np.asarray(getattr(b, name)), g['t_' + name], rtol=0, atol=1e-13, err_msg=name)
    np.testing.assert_allclose(b.transform, g['transform'], atol=1e-14)
    np.testing.assert_array_equal(b.exchange_sign, g['exchange_sign'])


def test_bipolar_isometry_exchange_and_subsets():
    g, b = build()
    U = b.transform
    np.testing.assert_allclose(U.T @ U, np.eye(b.nc), atol=1e-12)
    x = np.random.default_rng(3).normal(size=b.size) + 0j
    np.testing.assert_allclose(b.project(b.expand(x)), x, atol=1e-12)
    # one total M and the natural-parity subset are sub-bases of the full one
    _, b0 = build(M=0)
    assert all(c[3] == 0 for c in b0.basis) and set(b0.basis) <= set(b.basis)
    _, bn = build(natural_parity=True)
    assert all((l + j - L) % 2 == 0 for l, j, L, _ in bn.basis)
    assert b0.transform.shape[0] == sum(1 for a, c in b.uncoupled.ch if a[1] + c[1] == 0)
