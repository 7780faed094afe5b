"""Device backward propagation of the He+ channel functions (laqphysics_b200.ionic_adjoint)
against the reference's sparse-LU CF4 propagation of the same duals
(tests/golden/ionic_adjoint.npz from python/streaming_surface.py:125-146), and the
operator / preconditioner against scipy on the host.

Tolerances: operator 1e-13 relative; preconditioner inverse 1e-10; channel functions
1e-10 relative L2 at every step (GMRES to 1e-12 per solve against exact LU solves)."""
import json

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'


def ionic_case():
    from laqphysics_b200.fedvr import make_grid
    from laqphysics_b200.helium3d import Helium
    from laqphysics_b200.pulses import Pulse
    from laqphysics_b200.surface3d import Ionic
    g = golden('ionic_adjoint')
    base = Helium(make_grid(**json.loads(str(g['grid']))), 1, M=0, cutoff_radii=tuple(g['cutoff']))
    ion = Ionic(base, {0})
    pulse = Pulse(**json.loads(str(g['pulse'])))
    avec = lambda t: np.array([0., 0., float(pulse.vector(t))])
    return g, ion, avec


def test_ionic_operator_and_preconditioner():
    from laqphysics_b200.ionic_adjoint import IonicAdjoint
    g, ion, _ = ionic_case()
    engine = IonicAdjoint(ion, 3, DEVICE)
    rng = np.random.default_rng(2)
    X = rng.normal(size=(engine.ndof, 3)) + 1j * rng.normal(size=(engine.ndof, 3))
    A = np.array([.03, -.02, .15])
    ref = ion.matrix(A).conj().T @ X
    y = engine.host(engine.apply(engine.tensor(X), engine.coefficients(A)))
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-13
    alpha, e_ref = .05 / (3 + 1j * np.sqrt(3)), -1.7
    x = engine.tensor(X)
    back = engine.precondition(engine.apply_shifted(x, np.zeros(4), alpha, e_ref), alpha, -e_ref)
    assert np.linalg.norm(engine.host(back) - X) / np.linalg.norm(X) < 1e-10


def test_channel_functions_match_reference_cf4():
    from laqphysics_b200.ionic_adjoint import channel_functions
    g, ion, avec = ionic_case()
    unique = [tuple(int(v) for v in u) for u in g['unique']]
    states = g['states']
    steps = len(states) - 1
    dt, t_end = float(g['dt']), float(g['t_end'])
    times = t_end - dt * np.arange(steps, -1, -1)
    chi = channel_functions(ion, unique, avec, times, DEVICE).cpu().numpy()
    for k in range(steps + 1):   # golden k = k steps back from t_end
        got = chi[steps - k]
        assert np.linalg.norm(got - states[k]) / np.linalg.norm(states[k]) < 1e-10, k
