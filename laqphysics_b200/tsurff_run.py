"""A channel-resolved tSURFF propagation on the device: velocity-gauge Arnoldi steps of
the two-electron state, a surface sample after every step (flux frame, ionic contraction,
Volkov accumulation), and the spectrum at the end.

This strings together the pieces the reference's driver strings together in
python/run3d.py:181-224 with the online extraction of python/streaming_surface.py:185-278,
so that a complex128 run and a mixed-precision run (complex64 H·psi inside the complex128
Krylov, every surface quantity in complex128) can be compared on equal terms.

The ionic channel functions chi_c(t) are the dual final He+ states propagated backward
with the ionic Hamiltonian, chi(t_k) = exp(+i dt H_ion(A(t_k + dt/2))^dagger) chi(t_{k+1})
(python/streaming_surface.py:125-146 propagates the same duals backward with CF4); they
are computed once on the host (scipy) and shared by every run.
"""
import numpy as np
import torch
from scipy.sparse.linalg import expm_multiply

from .streaming_surface import SurfaceSampler, VolkovAccumulator
from .torch_backend import FieldSchedule, step


def ionic_channel_functions(ion, unique, avec, dt, steps):
    """chi at t_k = k dt, k = 0..steps: (steps+1, na*n, len(unique)) complex."""
    chi = np.zeros((steps + 1, ion.na * ion.n, len(unique)), complex)
    chi[steps] = ion.dual_final_states(unique)
    for k in range(steps - 1, -1, -1):
        H = ion.matrix(avec((k + 0.5) * dt))
        chi[k] = expm_multiply(1j * dt * H.conj().T, chi[k + 1])
    return chi


def run(engine, contractor, config, psi0, avec, dt, steps, chi, precision='complex128', tol=1e-10, maxdim=16):
    """Propagate psi0 for `steps` velocity-gauge steps of dt, sampling the surface at every
    step; returns (accumulator, final state, mean Krylov dimension)."""
    acc = VolkovAccumulator(contractor, config, avec, device=engine.device)
    sampler = SurfaceSampler(engine, contractor, acc)
    schedule = FieldSchedule(engine, avec, velocity=True, precision=precision)
    psi = psi0.clone() if torch.is_tensor(psi0) else engine.state(psi0)
    sampler.record(0, 0.0, psi, avec(0.0), chi[0])
    dims = []
    for k in range(steps):
        psi, info = step(schedule, psi, k * dt, dt, tol, maxdim)
        dims.append(info['dimension'])
        sampler.record(k + 1, (k + 1) * dt, psi, avec((k + 1) * dt), chi[k + 1])
    return acc, psi, float(np.mean(dims))


def spectrum_error(acc_test, acc_ref):
    """Relative L2 difference of the angle-resolved photoelectron spectra (all labels,
    energies, directions) and the largest per-label angle-integrated difference."""
    pes_t, tot_t = acc_test.spectrum()
    pes_r, tot_r = acc_ref.spectrum()
    rel = float(np.linalg.norm(pes_t - pes_r) / np.linalg.norm(pes_r))
    per_label = float(np.max(np.linalg.norm(tot_t - tot_r, axis=1) / np.linalg.norm(tot_r, axis=1)))
    return rel, per_label
