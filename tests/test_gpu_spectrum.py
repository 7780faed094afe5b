"""Mixed precision against complex128 on a whole channel-resolved tSURFF run: velocity-
gauge Arnoldi propagation from the ground state through a short pulse, a surface sample
every step, He+ (n <= 2) channel spectra.  The mixed run applies H·psi in complex64 inside
the complex128 Krylov; everything on the surface stays complex128.

Stated tolerances (mixed vs complex128): photoelectron spectrum relative L2 error <= 1e-5,
final-state relative L2 error <= 1e-5, norm difference <= 1e-7."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'

CONFIG = {'radial': {'edges': [0, 1, 2, 3, 4, 6, 8, 10, 12], 'order': 4, 'tail': 8, 'ecs_angle': .3},
          'lmax': 1, 'M': 0, 'total_Lmax': 1, 'cutoff_radii': [3, 4], 'surface': 8.,
          'pulses': [{'pulse': {'omega': 2.0, 'cycles': 2, 'field': .3}, 'polarization': 'z'}],
          'ionic_channels': [[1, 0, 0], [2, 0, 0], [2, 1, 0]],
          'spectrum_energy': [.3, 2.3, 21], 'spectrum': {'theta_points': 4, 'phi_points': 1}}


def test_mixed_precision_tsurff_spectrum_against_complex128():
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.pulses import Pulse
    from laqphysics_b200.surface3d import Ionic
    from laqphysics_b200.surface_contract import SurfaceContractor
    from laqphysics_b200.tsurff_run import ionic_channel_functions, run, spectrum_error
    from laqphysics_b200.workloads import coupled
    rc = CONFIG['radial']
    build = lambda angle: coupled(rc['edges'], rc['order'], CONFIG['lmax'], CONFIG['total_Lmax'], ecs_angle=angle,
                                  tail=rc['tail'], cutoff_radii=tuple(CONFIG['cutoff_radii']))
    h, hreal = build(rc['ecs_angle']), build(0.)
    base = h.uncoupled
    base.prepare_surface(CONFIG['surface'])
    h.prepare_surface(CONFIG['surface'])
    labels = [tuple(x) for x in CONFIG['ionic_channels']]
    unique = list(dict.fromkeys((n, l, abs(m)) for n, l, m in labels))
    columns = [unique.index((n, l, abs(m))) for n, l, m in labels]
    ion = Ionic(base, {m for n, l, m in unique})
    contractor = SurfaceContractor(base, ion, labels, unique, columns, True, h.transform, DEVICE)
    pulse = Pulse(**CONFIG['pulses'][0]['pulse'])
    avec = lambda t: np.array([0., 0., float(pulse.vector(t))])
    _, g, _ = hreal.ground(tol=1e-10)
    ratio = np.sqrt(h.grid.weights / hreal.grid.weights)
    psi0 = (g.reshape(h.shape, order='F') * ratio[:, None, None] * ratio[None, :, None]).ravel(order='F')
    engine = B200Hamiltonian(h, DEVICE)
    dt = .02
    steps = int(round(pulse.duration / dt)) + 50   # the pulse and 1 a.u. after it
    chi = ionic_channel_functions(ion, unique, avec, dt, steps)
    acc64, psi64, _ = run(engine, contractor, CONFIG, psi0, avec, dt, steps, chi, 'complex128')
    acc32, psi32, _ = run(engine, contractor, CONFIG, psi0, avec, dt, steps, chi, 'mixed')
    rel, per_label = spectrum_error(acc32, acc64)
    pes, _ = acc64.spectrum()
    assert np.isfinite(pes).all() and pes.max() > 0
    assert rel <= 1e-5, rel
    state = float(torch.linalg.vector_norm(psi32 - psi64) / torch.linalg.vector_norm(psi64))
    assert state <= 1e-5, state
    assert abs(float(torch.linalg.vector_norm(psi32)) - float(torch.linalg.vector_norm(psi64))) <= 1e-7
