"""Online channel-resolved tSURFF accumulation on the device (complex128).

Restates, with the reference's call surface:

* ``energy_grid`` / ``directions`` (python/streaming_surface.py:26-37): the spectral
  energy grid and the Gauss-Legendre x uniform-phi angular quadrature;
* ``VolkovAccumulator`` (python/streaming_surface.py:39-82, GPU twin :84-123): Volkov
  test functions j_l(k r) sqrt(w) r sqrt(2/pi) (-i)^l, harmonics Y_lm, the trapezoid
  integral of i sqrt(2) (radial @ harmonics) exp(i (E t + k u.int A + int A^2 / 2));
  ``add`` runs one device launch per surface sample, the amplitude never leaves the
  device until ``payload``/``write``;
* ``SurfaceSampler``: flux frame -> ionic contraction -> Volkov accumulation for one
  surface sample, entirely on the device (no host copy of the frame).
"""
import ctypes as ct

import numpy as np
import torch
from scipy.special import sph_harm_y, spherical_jn

from ._lib import LIB, check


def directions(config):
    s = config.get('spectrum', {})
    axial = config.get('M', 0) == 0
    nt = int(s.get('theta_points', 24 if not axial else 32))
    nf = int(s.get('phi_points', 1 if axial else 32))
    if nt < 2 or nf < 1 or (not axial and nf < 2):
        raise ValueError('invalid angular quadrature')
    z, w = np.polynomial.legendre.leggauss(nt)
    t, p = np.meshgrid(np.arccos(z), np.arange(nf) * 2 * np.pi / nf, indexing='ij')
    return t.ravel(), p.ravel(), np.repeat(w, nf) * 2 * np.pi / nf


def energy_grid(config):
    segments = config.get('spectrum', {}).get('energy_segments')
    if segments:
        result = np.unique(np.concatenate([np.linspace(float(a), float(b), int(n)) for a, b, n in segments]))
    else:
        result = np.linspace(*config.get('spectrum_energy', [.01, 1., 397]))
    if len(result) < 3 or np.any(result <= 0) or not np.isfinite(result).all():
        raise ValueError('invalid positive energy grid')
    return result


class VolkovAccumulator:
    def __init__(self, contractor, config, avec, max_file_bytes=None, device='cuda:0'):
        h = contractor.h
        self.labels = contractor.labels
        self.avec = avec
        self.device = torch.device(device)
        self.energy = energy_grid(config)
        self.k = np.sqrt(2 * self.energy)
        self.theta, self.phi, self.solid_angle_weights = directions(config)
        self.unit = np.array([np.sin(self.theta) * np.cos(self.phi), np.sin(self.theta) * np.sin(self.phi),
                              np.cos(self.theta)]).T
        r = h.r[h.surface_indices].real
        w = h.grid.weights[h.surface_indices].real
        self.outerstates = contractor.outerstates
        self.tests = np.array([np.sqrt(2 / np.pi) * (-1j) ** l * np.sqrt(w)[None, :] * r[None, :] *
                               spherical_jn(l, self.k[:, None] * r[None, :]) for l, m in self.outerstates])
        self.harmonics = np.array([sph_harm_y(l, m, self.theta, self.phi) for l, m in self.outerstates])
        shape = (len(self.labels), len(self.energy), len(self.theta))
        dev = lambda a, dt=torch.complex128: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=self.device)
        self.amplitude = torch.zeros(shape, dtype=torch.complex128, device=self.device)
        self.previous = torch.zeros_like(self.amplitude)
        self._tests, self._harm = dev(self.tests), dev(self.harmonics)
        self._energy, self._k = dev(self.energy, torch.float64), dev(self.k, torch.float64)
        self._unit = dev(self.unit, torch.float64)
        self.intA = np.zeros(3)
        self.intA2 = 0.
        self.time = 0.
        self.index = -1

    @torch.no_grad()
    def add(self, index, time, q):
        """Accumulate one sample; q: (labels, outer, ns) complex128 (device tensor or numpy)."""
        if index != self.index + 1:
            raise ValueError('nonsequential spectrum samples')
        if self.index >= 0:
            d = time - self.time
            before, after = np.asarray(self.avec(self.time), float), np.asarray(self.avec(time), float)
            self.intA = self.intA + d * (before + after) / 2
            self.intA2 += d * (np.dot(before, before) + np.dot(after, after)) / 2
        else:
            d = 0.
        if not torch.is_tensor(q):
            q = torch.as_tensor(np.ascontiguousarray(q, dtype=complex), device=self.device)
        q = q.contiguous()
        nlab, ne, nang = self.amplitude.shape
        intA = np.ascontiguousarray(self.intA, dtype=np.float64)
        vp = lambda t: ct.c_void_p(t.data_ptr())
        check(LIB.he_volkov_add(nlab, len(self.outerstates), q.shape[2], ne, nang, vp(q), vp(self._tests),
                                vp(self._harm), vp(self._energy), vp(self._k), vp(self._unit), float(time),
                                intA.ctypes.data, float(self.intA2), float(d), int(self.index < 0), vp(self.amplitude),
                                vp(self.previous), ct.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)),
              'he_volkov_add')
        self.time = float(time)
        self.index = int(index)

    def payload(self):
        return {'amplitude': self.amplitude.cpu().numpy(), 'previous_integrand': self.previous.cpu().numpy(),
                'intA': self.intA.copy(), 'intA2': self.intA2, 'time': self.time, 'sample_index': self.index}

    def restore(self, data):
        dev = lambda a: torch.as_tensor(np.array(a, dtype=complex), device=self.device)
        self.amplitude, self.previous = dev(data['amplitude']), dev(data['previous_integrand'])
        self.intA = np.array(data['intA'], float)
        self.intA2, self.time, self.index = float(data['intA2']), float(data['time']), int(data['sample_index'])

    def spectrum(self):
        """(pes, angle-integrated) as in the reference's write(): |b|^2 k and its solid-angle sum."""
        amp = self.amplitude.cpu().numpy()
        pes = abs(amp) ** 2 * self.k[None, :, None]
        return pes, np.sum(pes * self.solid_angle_weights[None, None, :], axis=2)

    def write(self, path, signature='', max_file_bytes=4_000_000_000):
        """The spectrum file of python/streaming_surface.py:74-82 (same keys, atomic capped write)."""
        from .checkpoint import capped_npz
        pes, total = self.spectrum()
        capped_npz(path, max_file_bytes, energy=self.energy, theta=self.theta, phi=self.phi,
                   solid_angle_weights=self.solid_angle_weights, amplitudes=self.amplitude.cpu().numpy(), pes=pes,
                   angle_integrated=total, labels=self.labels, source_signature=signature,
                   extraction_end_time=self.time, projection_final_time=self.time,
                   spectrum_scope='single ionization into the explicitly recorded bound ionic channels',
                   angular_rule='gauss', storage_method='online device accumulation')


TorchVolkovAccumulator = VolkovAccumulator


class SurfaceSampler:
    """One tSURFF surface sample on the device: flux frame (engine), ionic contraction
    with the device channel functions chi, Volkov accumulation.  Optional storage in the
    reference's sharded layout (surface_storage.ShardedArray): `projected` keeps q of every
    sample (storage mode 'projected', python/streaming_surface.py:255), `raw` the flux frame
    (mode 'raw_shards', python/run3d.py:139-141)."""

    def __init__(self, engine, contractor, accumulator, projected=None, raw=None):
        self.engine, self.contractor, self.accumulator = engine, contractor, accumulator
        self.projected, self.raw = projected, raw

    @torch.no_grad()
    def record(self, index, time, state, field, chi):
        frame = self.engine.surface.frame(state, field)
        if self.raw is not None:
            self.raw[index] = frame
        if not torch.is_tensor(chi):
            chi = torch.as_tensor(np.ascontiguousarray(chi, dtype=complex), device=self.engine.device)
        q = self.contractor.contract(chi, frame)
        self.accumulator.add(index, time, q)
        if self.projected is not None:
            self.projected[index] = q
        return q
