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
  surface sample, entirely on the device (no host copy of the frame), by default in one
  launch (``FusedSample``).
"""
import ctypes as ct

import numpy as np
import torch
from scipy.special import sph_harm_y, spherical_jn

from ._lib import HE_ERR_SHAPE, LIB, HeliumError, check


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
        self._last_a = None   # (time, A(time)) of the latest sample
        self.time = 0.
        self.index = -1

    def _advance(self, index, time):
        """Trapezoid bookkeeping of a new sample (int A, int A^2 up to `time`): returns the
        step d and whether this is the first sample."""
        if index != self.index + 1:
            raise ValueError('nonsequential spectrum samples')
        if self.index >= 0:
            d = time - self.time
            cached = self._last_a
            before = cached[1] if cached is not None and cached[0] == self.time else \
                np.asarray(self.avec(self.time), float)
            after = np.asarray(self.avec(time), float)
            self._last_a = (float(time), after)
            self.intA = self.intA + d * (before + after) / 2
            self.intA2 += d * (np.dot(before, before) + np.dot(after, after)) / 2
        else:
            d = 0.
        return float(d), int(self.index < 0)

    def _commit(self, index, time):
        self.time = float(time)
        self.index = int(index)

    @torch.no_grad()
    def add(self, index, time, q):
        """Accumulate one sample; q: (labels, outer, ns) complex128 (device tensor or numpy)."""
        d, first = self._advance(index, time)
        if not torch.is_tensor(q):
            q = torch.as_tensor(np.ascontiguousarray(q, dtype=complex), device=self.device)
        q = q.contiguous()
        nlab, ne, nang = self.amplitude.shape
        intA = np.ascontiguousarray(self.intA, dtype=np.float64)
        vp = lambda t: ct.c_void_p(t.data_ptr())
        check(LIB.he_volkov_add(nlab, len(self.outerstates), q.shape[2], ne, nang, vp(q), vp(self._tests),
                                vp(self._harm), vp(self._energy), vp(self._k), vp(self._unit), float(time),
                                intA.ctypes.data, float(self.intA2), float(d), first, vp(self.amplitude),
                                vp(self.previous), ct.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)),
              'he_volkov_add')
        self._commit(index, time)

    def payload(self):
        return {'amplitude': self.amplitude.cpu().numpy(), 'previous_integrand': self.previous.cpu().numpy(),
                'intA': self.intA.copy(), 'intA2': self.intA2, 'time': self.time, 'sample_index': self.index}

    def restore(self, data):
        dev = lambda a: torch.as_tensor(np.array(a, dtype=complex), device=self.device)
        self.amplitude, self.previous = dev(data['amplitude']), dev(data['previous_integrand'])
        self.intA = np.array(data['intA'], float)
        self.intA2, self.time, self.index = float(data['intA2']), float(data['time']), int(data['sample_index'])
        self._last_a = None

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


class FusedSample:
    """The device tables of one surface sample launch (he_sample_create): the engine's flux
    stencil window, the contractor's entry lists and the accumulator's Volkov tables."""

    def __init__(self, engine, contractor, accumulator):
        flux = engine.surface
        nlab, nouter, ns = contractor.shape
        if flux.ns != ns:
            raise ValueError('surface stencil rows and contraction rows differ')
        nlab_acc, ne, nang = accumulator.amplitude.shape
        vp = lambda t: ct.c_void_p(t.data_ptr())
        handle = ct.c_void_p()
        check(LIB.he_sample_create(ct.byref(handle), engine.op.handle, ns, flux.lo, flux.width, vp(flux.J),
                                   vp(flux.JP), len(contractor.unique), nlab, nouter, vp(contractor._eptr),
                                   vp(contractor._ecol), vp(contractor._einner), vp(contractor._ecoef),
                                   vp(contractor._eouter), vp(contractor._column), ne, nang, vp(accumulator._tests),
                                   vp(accumulator._harm), vp(accumulator._energy), vp(accumulator._k),
                                   vp(accumulator._unit)), 'he_sample_create')
        self.handle = handle
        self.grid = LIB.he_sample_grid(handle)
        self.tables = (flux, contractor, accumulator)   # the device arrays the handle reads

    def status(self):
        check(LIB.he_sample_status(self.handle), 'he_sample_status')

    def __del__(self):
        if getattr(self, 'handle', None):
            LIB.he_sample_destroy(self.handle)
            self.handle = None


class SurfaceSampler:
    """One tSURFF surface sample on the device: flux frame (engine), ionic contraction
    with the device channel functions chi, Volkov accumulation.  By default the three run
    as one launch (``FusedSample``, he_sample_record); ``fused=False``, or a surface beyond
    that launch's limits, runs them as three (he_flux, he_surface_contract, he_volkov_add).  Optional storage in the reference's
    sharded layout (surface_storage.ShardedArray): `projected` keeps q of every sample
    (storage mode 'projected', python/streaming_surface.py:255), `raw` the flux frame (mode
    'raw_shards', python/run3d.py:139-141)."""

    def __init__(self, engine, contractor, accumulator, projected=None, raw=None, fused=True):
        self.engine, self.contractor, self.accumulator = engine, contractor, accumulator
        self.projected, self.raw = projected, raw
        self.fused = None
        # the one launch recomputes SurfaceFlux's frame; an engine with another surface
        # object keeps the three launches, which call its own frame()
        from .surface import SurfaceFlux
        if fused and type(getattr(engine, 'surface', None)) is SurfaceFlux:
            try:
                self.fused = FusedSample(engine, contractor, accumulator)
            except HeliumError as error:
                # beyond the one-launch limits (more than 16 surface rows or 1024 contracted
                # values per sample): the three launches serve any size
                if error.status != HE_ERR_SHAPE:
                    raise

    @torch.no_grad()
    def record(self, index, time, state, field, chi):
        if not torch.is_tensor(chi):
            chi = torch.as_tensor(np.ascontiguousarray(chi, dtype=complex), device=self.engine.device)
        if self.fused is None:
            frame = self.engine.surface.frame(state, field)
            q = self.contractor.contract(chi, frame)
            self.accumulator.add(index, time, q)
        else:
            frame, q = self._record_fused(index, time, state, field, chi)
        if self.raw is not None:
            self.raw[index] = frame
        if self.projected is not None:
            self.projected[index] = q
        return q

    def _record_fused(self, index, time, state, field, chi):
        e, acc = self.engine, self.accumulator
        e._check(state, torch.complex128)
        ns = self.contractor.shape[2]
        frame = torch.empty((e.nc, ns, e.n), dtype=torch.complex128, device=e.device)
        q = torch.empty(self.contractor.shape, dtype=torch.complex128, device=e.device)
        chi = chi.contiguous()
        d, first = acc._advance(index, time)
        f = np.ascontiguousarray(field, dtype=np.float64)
        intA = np.ascontiguousarray(acc.intA, dtype=np.float64)
        vp = lambda t: ct.c_void_p(t.data_ptr())
        check(LIB.he_sample_record(self.fused.handle, vp(state), vp(chi), f.ctypes.data, float(time), intA.ctypes.data,
                                   float(acc.intA2), d, first, vp(frame), vp(q), vp(acc.amplitude), vp(acc.previous),
                                   ct.c_void_p(torch.cuda.current_stream(e.device).cuda_stream)), 'he_sample_record')
        acc._commit(index, time)
        return frame.permute(2, 1, 0), q
