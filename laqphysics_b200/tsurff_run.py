"""A channel-resolved tSURFF propagation on the device: velocity-gauge Arnoldi steps of
the two-electron state, a surface sample after every step (flux frame, ionic contraction,
Volkov accumulation), and the spectrum at the end.

This strings together the pieces the reference's driver strings together in
python/run3d.py:181-224 with the online extraction of python/streaming_surface.py:185-278,
so that a complex128 run and a mixed-precision run (complex64 H·psi inside the complex128
Krylov, every surface quantity in complex128) can be compared on equal terms.

The ionic channel functions chi_c(t) are the dual final He+ states propagated backward
with the adjoint ionic Hamiltonian by the reference's CF4 formula
(python/streaming_surface.py:125-146), on the device (laqphysics_b200.ionic_adjoint); they
are computed once per run and shared by the complex128 and mixed-precision runs.
"""
import numpy as np
import torch

from .ionic_adjoint import channel_functions
from .streaming_surface import SurfaceSampler, VolkovAccumulator
from .torch_backend import FieldSchedule, step


def ionic_channel_functions(ion, unique, avec, dt, steps, device='cuda:0'):
    """chi at t_k = k dt, k = 0..steps: device tensor (steps+1, na*n, len(unique))."""
    return channel_functions(ion, unique, avec, dt * np.arange(steps + 1), device)


def run(engine, contractor, config, psi0, avec, dt, steps, chi, precision='complex128', tol=1e-10, maxdim=16, t0=0.,
        fused=True):
    """Propagate psi0 from t0 for `steps` velocity-gauge steps of dt, sampling the surface
    at every step (chi[k] = channel functions at t0 + k dt; one launch per sample unless
    fused=False); returns (accumulator, final state, mean Krylov dimension)."""
    acc = VolkovAccumulator(contractor, config, avec, device=engine.device)
    sampler = SurfaceSampler(engine, contractor, acc, fused=fused)
    schedule = FieldSchedule(engine, avec, velocity=True, precision=precision)
    psi = psi0.clone() if torch.is_tensor(psi0) else engine.state(psi0)
    sampler.record(0, t0, psi, avec(t0), chi[0])
    dims = []
    for k in range(steps):
        psi, info = step(schedule, psi, t0 + k * dt, dt, tol, maxdim)
        dims.append(info['dimension'])
        t = t0 + (k + 1) * dt
        sampler.record(k + 1, t, psi, avec(t), chi[k + 1])
    return acc, psi, float(np.mean(dims))


def spectrum_error(acc_test, acc_ref):
    """Relative L2 difference of the angle-resolved photoelectron spectra (all labels,
    energies, directions) and the largest per-label angle-integrated difference."""
    pes_t, tot_t = acc_test.spectrum()
    pes_r, tot_r = acc_ref.spectrum()
    rel = float(np.linalg.norm(pes_t - pes_r) / np.linalg.norm(pes_r))
    per_label = float(np.max(np.linalg.norm(tot_t - tot_r, axis=1) / np.linalg.norm(tot_r, axis=1)))
    return rel, per_label


# A small channel-resolved case (the spectrum test and the bench's spectrum leg):
# 8 elements of order 4 to 12 a.u. + 8-point ECS tail, coupled l <= 1, L <= 1, surface at
# 8 a.u., 2-cycle sin^2 pulse omega 2.0 a.u. with peak field 0.3 a.u., He+ n <= 2 labels.
SMALL_CASE = {'radial': {'edges': [0, 1, 2, 3, 4, 6, 8, 10, 12], 'order': 4, 'tail': 8, 'ecs_angle': .3},
              'lmax': 1, 'M': 0, 'total_Lmax': 1, 'cutoff_radii': [3, 4], 'surface': 8.,
              'pulses': [{'pulse': {'omega': 2.0, 'cycles': 2, 'field': .3}, 'polarization': 'z'}],
              'ionic_channels': [[1, 0, 0], [2, 0, 0], [2, 1, 0]],
              'spectrum_energy': [.3, 2.3, 21], 'spectrum': {'theta_points': 4, 'phi_points': 1}}


def build_case(config, device, dt=.02, after=1.0, ground=None):
    """Engine, contractor, initial state (scaled ground state, python/run3d.py:134-136),
    vector potential, step count (pulse + `after` a.u.) and channel functions of a config.
    ``ground``: the real-grid ground state to start from (default: solved here on the
    device)."""
    from .engine import B200Hamiltonian
    from .pulses import Pulse
    from .surface3d import Ionic
    from .surface_contract import SurfaceContractor
    from .workloads import coupled
    rc = config['radial']
    build = lambda angle: coupled(rc['edges'], rc['order'], config['lmax'], config['total_Lmax'], ecs_angle=angle,
                                  tail=rc['tail'], cutoff_radii=tuple(config['cutoff_radii']))
    h, hreal = build(rc['ecs_angle']), build(0.)
    base = h.uncoupled
    base.prepare_surface(config['surface'])
    h.prepare_surface(config['surface'])
    labels = [tuple(x) for x in config['ionic_channels']]
    unique = list(dict.fromkeys((n, l, abs(m)) for n, l, m in labels))
    columns = [unique.index((n, l, abs(m))) for n, l, m in labels]
    ion = Ionic(base, {m for n, l, m in unique})
    contractor = SurfaceContractor(base, ion, labels, unique, columns, True, h.transform, device)
    pulse = Pulse(**config['pulses'][0]['pulse'])
    avec = lambda t: np.array([0., 0., float(pulse.vector(t))])
    g = ground if ground is not None else hreal.ground(tol=1e-10)[1]
    ratio = np.sqrt(h.grid.weights / hreal.grid.weights)
    psi0 = (g.reshape(h.shape, order='F') * ratio[:, None, None] * ratio[None, :, None]).ravel(order='F')
    engine = B200Hamiltonian(h, device)
    steps = int(round((pulse.duration + after) / dt))
    chi = ionic_channel_functions(ion, unique, avec, dt, steps, device)
    return engine, contractor, psi0, avec, steps, chi
