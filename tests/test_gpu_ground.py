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
