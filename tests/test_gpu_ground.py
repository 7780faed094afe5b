"""Ground state (python/ground_s.py:55-89) with the matvec on the GPU through the C-ABI
tensor_apply: energy and state agree with the reference's LOBPCG on the same grid."""
import json

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_ground_state_matches_reference():
    from laqphysics_b200.coupled_angular import CoupledHelium
    from laqphysics_b200.fedvr import make_grid
    from laqphysics_b200.helium3d import Helium
    g = golden('ground')
    u = Helium(make_grid(**json.loads(str(g['grid']))), int(g['lmax']), M=0)
    E, state, res = CoupledHelium(u, 2).ground(tol=1e-10)
    assert abs(E - float(g['energy'])) < 1e-9
    assert abs(abs(np.vdot(state, g['state'])) - 1) < 1e-8
    assert res < 1e-6


def test_ground_only_representation_and_eigsh_agree_with_lobpcg():
    """GroundS.from_grid (python/ground_s.py:16-27, compressed state only) and the
    reference's eigsh alternative reach the device-LOBPCG energy of the same grid."""
    from laqphysics_b200.fedvr import make_grid
    from laqphysics_b200.ground_s import GroundS
    from laqphysics_b200.helium3d import Helium
    g = golden('ground')
    grid = make_grid(**json.loads(str(g['grid'])))
    lmax = int(g['lmax'])
    solver = GroundS.from_grid(grid, lmax)
    E, small, res = solver.solve(tol=1e-10)
    assert small.size == grid.r.size ** 2 * (lmax + 1)
    assert abs(E - float(g['energy'])) < 1e-9 and res < 1e-6
    assert 0 < solver.last_iterations < 250
    E2, _, _ = GroundS(Helium(grid, lmax, M=0)).solve(tol=1e-10, method='eigsh')
    assert abs(E2 - E) < 1e-9
