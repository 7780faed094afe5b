"""Host table builders reproduce the reference's grid, channel tables and pulses.

The device operator consumes these arrays, so they are compared to the
reference's own (golden fixtures from tests/golden/make_golden.py) entry by entry.
"""
import json

import numpy as np
import pytest

from conftest import golden
from laqphysics_b200.coupled_angular import CoupledHelium
from laqphysics_b200.fedvr import derivative, make_grid
from laqphysics_b200.helium3d import Helium
from laqphysics_b200.pulses import Pulse


@pytest.mark.parametrize('case', ['plain', 'ecs', 'ecs_cut', 'bridge', 'variable', 'long_tail'])
def test_grid_matches_reference(case):
    g = golden('grids')
    args = json.loads(str(g['cases']))[case]
    if isinstance(args.get('order'), list):
        args['order'] = tuple(args['order'])
    grid = make_grid(**args)
    np.testing.assert_allclose(grid.r, g[f'{case}_r'], rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(grid.weights, g[f'{case}_weights'], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(grid.kinetic.toarray(), g[f'{case}_kinetic'], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(grid.interior_weights, g[f'{case}_interior'], rtol=1e-14, atol=1e-15)


def test_grid_rejects_invalid_arguments():
    with pytest.raises(ValueError):
        make_grid([0, 1, 1], 3)
    with pytest.raises(ValueError):
        make_grid([0, 1, 2], 3, ecs_angle=.3)
    with pytest.raises(ValueError):
        make_grid([0, 1, 2], (3,))


def test_polynomial_derivative_is_exact():
    x = np.array([-1., -.4, .2, .8, 1.])
    np.testing.assert_allclose(derivative(x) @ (x ** 4), 4 * x ** 3, atol=1e-13)


def test_hydrogenic_energies_known_answer():
    from scipy.linalg import eigvalsh
    g = make_grid([0, .5, 1, 2, 4, 8, 16, 32], 8)
    for l in (0, 1, 2):
        e = eigvalsh(g.kinetic.toarray() + np.diag(-2 / g.r + l * (l + 1) / (2 * g.r * g.r)))
        np.testing.assert_allclose(e[0], -2 / (l + 1) ** 2, atol=2e-7)


def _compare_tables(h, g, rtol=1e-13):
    for name in ('ptr', 'col', 'vptr', 'vc', 'vl', 'dptr', 'dc', 'de', 'exchange'):
        np.testing.assert_array_equal(getattr(h, name), g['t_' + name], err_msg=name)
    for name in ('tv', 'diag', 'vcoef', 'rad', 'dcoef', 'ldiff', 'r'):
        np.testing.assert_allclose(getattr(h, name), g['t_' + name], rtol=rtol, atol=1e-13, err_msg=name)


def test_product_tables_match_reference():
    g = golden('apply_ecs')
    h = Helium(make_grid([0, .5, 1, 2, 4], 3, ecs_angle=.3, tail=5), 1, M=None)
    _compare_tables(h, g)
    d1, d2 = h.diag_parts
    np.testing.assert_array_equal(d1[:, None, :] + d2[None, :, :], h.diag)


def test_product_tables_with_cutoff_and_surface_match_reference():
    g = golden('apply_cut')
    h = Helium(make_grid([0, .5, 1, 2, 4, 6, 8], 3, ecs_angle=.4, tail=8), 1, M=None, cutoff_radii=[1, 2])
    _compare_tables(h, g)
    idx = h.prepare_surface(float(g['surface_radius']))
    np.testing.assert_array_equal(idx, g['surface_indices'])
    np.testing.assert_allclose(h.surface_T, g['surface_T'], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(h.surface_P, g['surface_P'], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(h.flux(g['x'], g['field']), g['flux'], rtol=1e-12, atol=1e-13)


def test_coupled_tables_match_reference():
    g = golden('apply_coupled')
    args = json.loads(str(g['grid']))
    u = Helium(make_grid(**args), 2, M=0, cutoff_radii=[1, 2])
    c = CoupledHelium(u, 2)
    _compare_tables(c, g)
    np.testing.assert_allclose(c.transform, g['transform'], atol=1e-15)
    np.testing.assert_array_equal(c.exchange_sign, g['exchange_sign'])
    c.prepare_surface(5)
    np.testing.assert_allclose(c.flux(g['x'], g['field']), g['flux'], rtol=1e-12, atol=1e-12)


def test_pulses_match_reference():
    g = golden('pulses')
    for k in range(3):
        p = Pulse(**json.loads(str(g[f'p{k}'])))
        np.testing.assert_allclose(p.electric(g['t']), g[f'p{k}_E'], rtol=1e-14, atol=1e-16)
        np.testing.assert_allclose(p.vector(g['t']), g[f'p{k}_A'], rtol=1e-13, atol=1e-16)
        # the scalar path of a time-step loop agrees with the array path
        scalar = np.array([p.vector(float(t)) for t in g['t']])
        np.testing.assert_allclose(scalar, g[f'p{k}_A'], rtol=1e-13, atol=1e-16)
