"""Mixed length/velocity gauge operator on the GPU (laqphysics_b200.mixed_gauge) against
the reference's MixedHamiltonian outputs (tests/golden/mixed_gauge.npz, python/
mixed_gauge.py:73-117 on CPU torch): a coupled M = 0 basis with a z field and a bipolar
all-M basis with a general (A, E) field.  Tolerance: rtol 2e-13, atol 2e-12 (the
reference's kernel bound); the shifted Pade operator against x + i alpha (H x - E x)."""
import json

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'


def operators():
    from laqphysics_b200.bipolar import BipolarHelium
    from laqphysics_b200.coupled_angular import CoupledHelium
    from laqphysics_b200.fedvr import make_grid
    from laqphysics_b200.helium3d import Helium
    g = golden('mixed_gauge')
    grid = make_grid(**json.loads(str(g['grid'])))
    cut = tuple(g['cutoff'])
    return g, {'coupled': CoupledHelium(Helium(grid, 2, M=0, cutoff_radii=cut), 2),
               'bipolar': BipolarHelium(grid, lmax=1, total_Lmax=2, M=None, cutoff_radii=cut)}


@pytest.mark.parametrize('case', ['coupled', 'bipolar'])
def test_mixed_gauge_apply_matches_reference(case):
    from laqphysics_b200.mixed_gauge import MixedB200Hamiltonian
    g, hs = operators()
    op = MixedB200Hamiltonian(hs[case], DEVICE, inner=float(g['inner']), outer=float(g['outer']))
    x = op.state(g[f'{case}_x'])
    for key, field in (('y', g[f'{case}_field']), ('y0', np.zeros(12))):
        y = op.host(op.apply(x, field))
        np.testing.assert_allclose(y, g[f'{case}_{key}'], rtol=2e-13, atol=2e-12, err_msg=key)
    alpha, e_ref = .05 / (3 + 1j * np.sqrt(3)), -2.9
    s = op.host(op.apply_shifted(x, g[f'{case}_field'], alpha, e_ref))
    ref = g[f'{case}_x'] + 1j * alpha * (g[f'{case}_y'] - e_ref * g[f'{case}_x'])
    np.testing.assert_allclose(s, ref, rtol=1e-12, atol=1e-12)
    op.synchronize()
