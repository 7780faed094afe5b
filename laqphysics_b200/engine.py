"""Device engine with the reference's ``TorchHamiltonian`` duck-type.

``B200Hamiltonian(h, device, coulomb_backend=...)`` can stand where the reference
constructs ``TorchHamiltonian(h, device, coulomb_backend=...)``
(python/run3d.py:189, python/torch_backend.py:11-138): the same attributes
(``n, nc, size, device, dtype, h, diagonal, coulomb_backend,
coulomb_block_bytes, a2_coefficient``) and methods (``state, host, synchronize,
apply, flux``), complex128 1-D contiguous states in the reference's Fortran order.
All arithmetic on states runs in this package's sm_100a kernels through the C-ABI
(include/helium_b200.h); torch only owns the device memory and the stream.
"""
import ctypes as ct

import numpy as np
import torch

from ._lib import HE_C64, HE_C128, LIB, HeliumError, check, ptr

PRECISIONS = {'complex128': (HE_C128, torch.complex128), 'complex64': (HE_C64, torch.complex64)}


def _host_tables(h):
    def arr(name, dtype):
        return np.ascontiguousarray(np.asarray(getattr(h, name)).ravel(order='F'), dtype=dtype)
    t = {name: arr(name, np.int32) for name in ('ptr', 'col', 'vptr', 'vc', 'vl', 'dptr', 'dc', 'de')}
    for name in ('tv', 'vcoef', 'r'):
        t[name] = arr(name, np.complex128)
    t['ldiff'] = arr('ldiff', np.float64)
    t['dcoef'] = np.ascontiguousarray(np.asarray(h.dcoef).reshape(3, -1).T, dtype=np.complex128)  # (nd, 3) rows
    t['rad'] = arr('rad', np.complex128)
    parts = getattr(h, 'diag_parts', None)
    if parts is not None:
        t['d1'] = np.ascontiguousarray(np.asarray(parts[0]).ravel(order='F'), dtype=np.complex128)
        t['d2'] = np.ascontiguousarray(np.asarray(parts[1]).ravel(order='F'), dtype=np.complex128)
        t['diag'] = None
    else:
        t['diag'] = arr('diag', np.complex128)
        t['d1'] = t['d2'] = None
    t['nlam'] = int(np.asarray(h.rad).shape[2]) if np.ndim(h.rad) == 3 else int(max(t['vl'], default=0) + 1)
    return t


def fp64_peaks(device='cuda:0', iters=4096):
    """Measured FP64 throughput of a device in TFLOP/s: {'dmma': tensor pipe (mma.sync
    m8n8k4 f64), 'dfma': FMA pipe} (he_fp64_peak)."""
    out = {}
    with torch.cuda.device(torch.device(device)):
        for kind, name in ((0, 'dmma'), (1, 'dfma')):
            v = ct.c_double()
            check(LIB.he_fp64_peak(kind, int(iters), ct.byref(v), _stream(torch.device(device))), 'he_fp64_peak')
            out[name] = v.value
    return out


class OperatorHandle:
    """Owns one ``he_handle`` (device tables) for a Hamiltonian table object ``h``."""

    def __init__(self, h, device, complex64=True):
        self.device = torch.device(device)
        if self.device.type != 'cuda':
            raise ValueError('the B200 engine runs on CUDA devices only')
        t = _host_tables(h)
        self._keep = t
        n, nc = int(h.n), int(h.nc)
        handle = ct.c_void_p()
        opt = lambda a: ptr(a) if a is not None else None
        with torch.cuda.device(self.device):
            status = LIB.he_create(ct.byref(handle), n, nc, len(t['tv']), ptr(t['ptr']), ptr(t['col']), ptr(t['tv']),
                                   opt(t['diag']), opt(t['d1']), opt(t['d2']), len(t['vc']), ptr(t['vptr']),
                                   ptr(t['vc']), ptr(t['vl']), ptr(t['vcoef']), ptr(t['rad']), t['nlam'],
                                   len(t['dc']), ptr(t['dptr']), ptr(t['dc']), ptr(t['de']), ptr(t['dcoef']),
                                   ptr(t['ldiff']), ptr(t['r']), 1 if complex64 else 0)
        check(status, 'he_create')
        self.handle = handle
        self.n, self.nc = n, nc

    def __del__(self):
        handle = getattr(self, 'handle', None)
        if handle is not None and handle.value:
            LIB.he_destroy(handle)
            self.handle = None


def _stream(device):
    return ct.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class B200Hamiltonian:
    """complex128 (or complex64) H·psi on one GPU with the TorchHamiltonian interface."""

    def __init__(self, h, device='cuda:0', angular_sparse=True, coulomb_backend='sparse', precision='complex128'):
        if coulomb_backend not in ('sparse', 'blocks'):
            raise ValueError('unknown Coulomb contraction')
        if precision not in PRECISIONS:
            raise ValueError('precision must be complex128 or complex64')
        self.h = h
        self.device = torch.device(device)
        self.n, self.nc, self.size = int(h.n), int(h.nc), int(h.size)
        self.dtype = torch.complex128
        self.precision = precision
        self.angular_sparse = angular_sparse
        # Multipoles are contracted on the fly in every mode: nothing is precomputed.
        self.coulomb_backend = coulomb_backend
        self.coulomb_block_bytes = 0
        self.a2_coefficient = 1.0
        self.op = OperatorHandle(h, self.device)
        self.diagonal = torch.empty(self.size, dtype=torch.complex128, device=self.device)
        check(LIB.he_diagonal(self.op.handle, ct.c_void_p(self.diagonal.data_ptr()), _stream(self.device)), 'he_diagonal')
        self.apply_count = 0
        info = (ct.c_longlong * 18)()
        check(LIB.he_info(self.op.handle, info, 18), 'he_info')
        self.tiled = bool(info[9])
        self.mix_blocks = {'complex128': 2, 'complex64': 4}
        self.band_stages = {'complex128': 1, 'complex64': 2}
        self.path = int(info[10])
        self.plan_info = {'elements': int(info[11]), 'tiles_per_axis': int(info[12]), 'groups': int(info[13]),
                          'wide_edges': int(info[14]), 'wide_dipole_edges': int(info[15]),
                          'band_kernel': bool(info[16]), 'kinetic_kernel': bool(info[17])}
        if hasattr(h, 'surface_indices'):
            self._prepare_flux()

    def use_tiled(self, flag=True):
        """Select the tiled kernels (default when the tables admit them) or the generic one."""
        self.set_path(1 if flag else 0)

    def set_path(self, path):
        """0: generic gather kernel; 1: tiled kernels with the TMA-staged kinetic kernel
        (default); 2: tiled kernels with the shared-memory radial kernel."""
        check(LIB.he_set_path(self.op.handle, int(path)), 'he_set_path')
        self.tiled = path != 0
        self.path = int(path)

    def kernels(self, precision='complex128'):
        """Names of the kernels one apply launches on the current path."""
        if not self.tiled:
            return ['hpsi_gather_kernel']
        if self.path == 2:
            radial = 'hpsi_radial_kernel'
        elif self.path == 1 and self.plan_info['band_kernel']:
            radial = 'hpsi_band_kernel'
        elif self.plan_info['kinetic_kernel']:
            radial = 'hpsi_kinetic_kernel'
        else:
            radial = 'hpsi_radial_kernel'
        return [radial, 'hpsi_mix_kernel']

    def set_mix_blocks(self, precision, blocks):
        """Register budget of the generated mixing kernel: sized for `blocks` CTAs of 128
        threads per SM (more CTAs, fewer registers per thread)."""
        check(LIB.he_set_mix_blocks(self.op.handle, PRECISIONS[precision][0], int(blocks)), 'he_set_mix_blocks')
        self.mix_blocks[precision] = int(blocks)

    def set_band_stages(self, precision, stages):
        """Length-gauge banded kinetic kernel of one precision: 2 TMA stages at one CTA per
        SM, or 1 stage with the registers of two CTAs per SM (same results)."""
        check(LIB.he_set_band_stages(self.op.handle, PRECISIONS[precision][0], int(stages)), 'he_set_band_stages')
        self.band_stages[precision] = int(stages)

    def _time_apply(self, x, out, field, velocity, precision, reps):
        for _ in range(2):
            self.apply(x, field, velocity, out=out, precision=precision)
        torch.cuda.synchronize(self.device)
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(reps):
            self.apply(x, field, velocity, out=out, precision=precision)
        stop.record()
        self.synchronize()
        return start.elapsed_time(stop) / reps

    @torch.no_grad()
    def autotune(self, field=(0., 0., .02), velocity=False, precisions=('complex128', 'complex64'),
                 candidates=(1, 2, 3, 4, 6), stages=(1, 2), reps=10, seed=0):
        """Pick, per precision, the launch shapes that give the fastest apply on this
        operator: the banded kinetic kernel's form (`stages`; length gauge only), then the
        mixing kernel's CTAs per SM (register budget).  Each candidate is compiled (or read
        from the kernel cache), warmed up and timed with CUDA events over `reps` applies of a
        seeded state; the fastest stays selected.  Returns {precision: {'band_stages':
        {stages: ms}, 'mix_blocks': {blocks: ms per apply}}}."""
        if not self.tiled:
            return {}
        rng = np.random.default_rng(seed)
        x128 = self.state(rng.normal(size=self.size) + 1j * rng.normal(size=self.size))
        timings = {}
        for precision in precisions:
            x = x128 if precision == 'complex128' else x128.to(torch.complex64)
            out = torch.empty_like(x)
            timings[precision] = {}
            if not velocity and stages:
                result = {}
                for st in stages:
                    self.set_band_stages(precision, st)
                    result[st] = self._time_apply(x, out, field, velocity, precision, reps)
                self.set_band_stages(precision, min(result, key=result.get))
                timings[precision]['band_stages'] = result
            result = {}
            for blocks in candidates:
                self.set_mix_blocks(precision, blocks)
                result[blocks] = self._time_apply(x, out, field, velocity, precision, reps)
            self.set_mix_blocks(precision, min(result, key=result.get))
            timings[precision]['mix_blocks'] = result
        return timings

    @property
    def launches_per_apply(self):
        """Kernels one apply launches: radial (kinetic) and channel mixing, or one generic."""
        return 2 if self.tiled else 1

    def device_status(self):
        """Wait for the device and raise if a bounded device-side wait ran out."""
        check(LIB.he_device_status(self.op.handle), 'device status')

    # --- state transfer -------------------------------------------------------------
    def state(self, x):
        return torch.as_tensor(np.array(np.asarray(x).ravel(), dtype=np.complex128, copy=True), device=self.device)

    def host(self, x):
        return x.detach().cpu().numpy()

    def synchronize(self):
        torch.cuda.synchronize(self.device)
        self.device_status()

    # --- run diagnostics (python/run3d.py:212-224) -------------------------------------
    def diagnostics(self, x, ground=None):
        """The driver's checkpoint diagnostics computed on the device (he_diagnostics),
        without copying the state to the host: {'real_region_norm': sum |u|^2 f_i f_j with
        f = interior weight / |weight| (the real-element mass fraction), 'ground_population':
        |<g|psi>|^2 (ground: device state, or None), 'exchange_error': ||u - P12 u||}."""
        self._check(x, torch.complex128)
        if ground is not None:
            self._check(ground, torch.complex128)
        if not hasattr(self, '_diag_tables'):
            g = self.h.grid
            f = np.asarray(g.interior_weights / np.abs(g.weights), dtype=np.float64)
            sign = np.asarray(getattr(self.h, 'exchange_sign', np.ones(self.nc)), dtype=np.float64)
            self._diag_tables = (torch.as_tensor(f, device=self.device),
                                 torch.as_tensor(np.asarray(self.h.exchange, dtype=np.int32), device=self.device),
                                 torch.as_tensor(sign, device=self.device))
        f, xc, sign = self._diag_tables
        out = (ct.c_double * 4)()
        vp = lambda t: ct.c_void_p(t.data_ptr())
        check(LIB.he_diagnostics(self.op.handle, vp(x), vp(ground) if ground is not None else None, vp(f), vp(xc),
                                 vp(sign), out, _stream(self.device)), 'he_diagnostics')
        return {'real_region_norm': out[0], 'ground_population': out[1] ** 2 + out[2] ** 2 if ground is not None else None,
                'exchange_error': out[3]}

    def _check(self, x, dtype):
        if x.device != self.device or x.dtype != dtype or not x.is_contiguous() or x.numel() != self.size:
            raise ValueError(f'state must be a contiguous {dtype} tensor of {self.size} elements on {self.device}')

    # --- operator -------------------------------------------------------------------
    @torch.no_grad()
    def apply(self, x, field=(0., 0., 0.), velocity=True, out=None, precision=None):
        """out = H(field) x; complex128 unless ``precision='complex64'`` (then x, out are complex64)."""
        code, dtype = PRECISIONS[precision or ('complex128' if x.dtype == torch.complex128 else 'complex64')]
        self._check(x, dtype)
        if out is None:
            out = torch.empty_like(x)
        f = np.ascontiguousarray(field, dtype=np.float64)
        if f.shape != (3,):
            raise ValueError('field must have three Cartesian components')
        check(LIB.he_apply(self.op.handle, ct.c_void_p(x.data_ptr()), ct.c_void_p(out.data_ptr()), ptr(f),
                           int(bool(velocity)), code, _stream(self.device)), 'he_apply')
        self.apply_count += 1
        return out

    @torch.no_grad()
    def apply_host_stream(self, xs, field=(0., 0., 0.), velocity=True, outs=None, precision=None):
        """outs[k] = H(field) xs[k] for a sequence of host states (pinned CPU tensors), with
        the transfers overlapped: while state k is applied, state k+1 is copied in on one
        stream and the result of state k-1 is copied out on another (the two directions use
        separate copy engines), through two device buffers each way.  Returns `outs`
        (allocated pinned when None) after the last copy has landed."""
        code, dtype = PRECISIONS[precision or ('complex128' if xs[0].dtype == torch.complex128 else 'complex64')]
        for x in xs:
            if x.device.type != 'cpu' or x.dtype != dtype or x.numel() != self.size:
                raise ValueError(f'host states must be {dtype} CPU tensors of {self.size} elements')
        if outs is None:
            outs = [torch.empty(self.size, dtype=dtype).pin_memory() for _ in xs]
        dev_in = [torch.empty(self.size, dtype=dtype, device=self.device) for _ in range(2)]
        dev_out = [torch.empty_like(dev_in[0]) for _ in range(2)]
        compute = torch.cuda.current_stream(self.device)
        h2d, d2h = torch.cuda.Stream(self.device), torch.cuda.Stream(self.device)
        h2d.wait_stream(compute)
        d2h.wait_stream(compute)
        loaded = [torch.cuda.Event() for _ in range(2)]
        applied = [torch.cuda.Event() for _ in range(2)]
        drained = [torch.cuda.Event() for _ in range(2)]
        for k, x in enumerate(xs):
            b = k % 2
            with torch.cuda.stream(h2d):
                if k >= 2:
                    h2d.wait_event(applied[b])      # state k-2 no longer reads dev_in[b]
                dev_in[b].copy_(x, non_blocking=True)
                loaded[b].record(h2d)
            compute.wait_event(loaded[b])
            if k >= 2:
                compute.wait_event(drained[b])      # result k-2 has left dev_out[b]
            self.apply(dev_in[b], field, velocity, out=dev_out[b], precision=precision)
            applied[b].record(compute)
            with torch.cuda.stream(d2h):
                d2h.wait_event(applied[b])
                outs[k].copy_(dev_out[b], non_blocking=True)
                drained[b].record(d2h)
        compute.wait_stream(d2h)
        compute.wait_stream(h2d)
        for t in dev_in + dev_out:
            t.record_stream(compute)
        torch.cuda.current_stream(self.device).synchronize()
        return outs

    @torch.no_grad()
    def apply_batched(self, x, fields, velocity=True, out=None, precision=None):
        """out[b] = H(fields[b]) x[b] for a batch of instances sharing this operator:
        x is (count, size) (or count*size) complex128/complex64, fields is (count, 3)."""
        code, dtype = PRECISIONS[precision or ('complex128' if x.dtype == torch.complex128 else 'complex64')]
        f = np.ascontiguousarray(fields, dtype=np.float64).reshape(-1, 3)
        count = f.shape[0]
        if x.device != self.device or x.dtype != dtype or not x.is_contiguous() or x.numel() != count * self.size:
            raise ValueError(f'batch must be a contiguous {dtype} tensor of {count} x {self.size} elements on {self.device}')
        if out is None:
            out = torch.empty_like(x)
        check(LIB.he_apply_batched(self.op.handle, count, ct.c_void_p(x.data_ptr()), ct.c_void_p(out.data_ptr()),
                                   ptr(f), int(bool(velocity)), code, _stream(self.device)), 'he_apply_batched')
        self.apply_count += count
        return out

    @torch.no_grad()
    def apply_shifted(self, x, field, alpha, reference_energy=0., velocity=True, out=None):
        """out = x + i*alpha*(H(field) x - E_ref x): the Pade operator of python/implicit.py:77-84."""
        code, dtype = PRECISIONS['complex128' if x.dtype == torch.complex128 else 'complex64']
        self._check(x, dtype)
        if out is None:
            out = torch.empty_like(x)
        f = np.ascontiguousarray(field, dtype=np.float64)
        alpha = complex(alpha)
        check(LIB.he_apply_shifted(self.op.handle, ct.c_void_p(x.data_ptr()), ct.c_void_p(out.data_ptr()), ptr(f),
                                   int(bool(velocity)), alpha.real, alpha.imag, float(reference_energy), code,
                                   _stream(self.device)), 'he_apply_shifted')
        self.apply_count += 1
        return out

    # --- surface flux ---------------------------------------------------------------
    def _prepare_flux(self):
        from .surface import SurfaceFlux
        self.surface = SurfaceFlux(self)

    @torch.no_grad()
    def flux(self, x, field):
        if not hasattr(self, 'surface'):
            if not hasattr(self.h, 'surface_indices'):
                raise HeliumError(1, 'prepare_surface() was not called on the Hamiltonian tables')
            self._prepare_flux()
        return self.host(self.surface.frame(x, field))


TorchHamiltonian = B200Hamiltonian
