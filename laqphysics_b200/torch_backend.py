"""Drop-in for the reference's python/torch_backend.py: ``TorchHamiltonian``,
``exponential_action`` and ``step`` with the same signatures, messages and results,
computed by this package's sm_100a kernels.

* ``TorchHamiltonian`` is :class:`laqphysics_b200.engine.B200Hamiltonian`.
* ``exponential_action(apply, x, dt, tol, maxdim)`` (python/torch_backend.py:140-158):
  Arnoldi with CGS2, the small Hessenberg exponential and the error estimate all on
  the device; ``apply`` may be any callable returning H·y.  The host waits only at the
  reference's check points (m = 4, 8, ..., maxdim), not once per Krylov vector.
  When ``apply`` is a :class:`FieldOperator` of this package the whole Krylov loop
  runs inside the C-ABI (``he_expv``) with no Python in between.
* ``step(apply_at, x, t, dt, tol, maxdim)`` (python/torch_backend.py:160-167): midpoint
  Hamiltonian, recursive dt halving (depth <= 8) on 'Arnoldi did not converge'.
"""
import ctypes as ct

import numpy as np
import torch

from ._lib import HE_ERR_NOCONV, LIB, HeliumError, check, ptr
from .engine import B200Hamiltonian, _stream

TorchHamiltonian = B200Hamiltonian

_WORKSPACES = {}
_GRAPHS = [True]


def use_cuda_graphs(flag=True):
    """Replay repeated Arnoldi solves (same operator, precision, gauge and maxdim as the
    previous solve on the workspace) as one captured CUDA graph (he_krylov_set_graphs; on
    by default); applies to existing and future workspaces.  Results are identical either
    way.  Returns the previous setting."""
    previous = _GRAPHS[0]
    _GRAPHS[0] = bool(flag)
    for ws in list(_WORKSPACES.values()) + list(_BATCHED.values()):
        check(LIB.he_krylov_set_graphs(ws.handle, int(flag)), 'he_krylov_set_graphs')
    return previous


class KrylovWorkspace:
    """Device Krylov basis (maxdim+1 vectors), Hessenberg matrix and reduction scratch."""

    def __init__(self, n, maxdim, device, flexible=False):
        self.n, self.maxdim, self.device = int(n), int(maxdim), torch.device(device)
        handle = ct.c_void_p()
        with torch.cuda.device(self.device):
            check(LIB.he_krylov_create(ct.byref(handle), self.n, self.maxdim, int(flexible)), 'he_krylov_create')
        self.handle = handle
        self._views = {}
        if _GRAPHS[0] and not flexible:
            check(LIB.he_krylov_set_graphs(handle, 1), 'he_krylov_set_graphs')

    def vector(self, j, which=0):
        """torch view of basis vector j (which=0: Q, which=1: Z of flexible GMRES)."""
        key = (which, j)
        if key not in self._views:
            address = ct.c_void_p()
            check(LIB.he_krylov_vector(self.handle, which, j, ct.byref(address)), 'he_krylov_vector')
            self._views[key] = _device_view(address.value, self.n, self.device)
        return self._views[key]

    def __del__(self):
        handle = getattr(self, 'handle', None)
        if handle is not None and handle.value:
            LIB.he_krylov_destroy(handle)
            self.handle = None


class _Owner:
    """Keeps a raw device allocation visible to torch without taking ownership."""

    def __init__(self, address, nbytes):
        self.__cuda_array_interface__ = {'shape': (nbytes // 16,), 'typestr': '<c16', 'data': (address, False),
                                         'version': 3, 'strides': None}


def _device_view(address, n, device):
    return torch.as_tensor(_Owner(address, n * 16), device=device)


def workspace(n, maxdim, device, flexible=False):
    """Cached workspace with at least ``maxdim`` Krylov vectors for vectors of length n, one
    per CUDA stream (solves running concurrently on different streams never share one)."""
    device = torch.device(device)
    key = (device, int(n), bool(flexible), torch.cuda.current_stream(device).cuda_stream)
    ws = _WORKSPACES.get(key)
    if ws is None or ws.maxdim < maxdim:
        ws = KrylovWorkspace(n, max(maxdim, ws.maxdim if ws else 0), device, flexible)
        _WORKSPACES[key] = ws
    return ws


class FieldOperator:
    """y -> H(field) y of a B200Hamiltonian; also usable as a plain callable.
    precision='mixed' runs H·psi in complex64 inside the fused Arnoldi (the Krylov basis,
    CGS2, the Hessenberg exponential and the error estimate stay complex128)."""

    def __init__(self, engine, field, velocity=True, precision='complex128'):
        if precision not in ('complex128', 'mixed'):
            raise ValueError("precision must be 'complex128' or 'mixed'")
        self.engine = engine
        self.field = np.ascontiguousarray(field, dtype=np.float64)
        self.velocity = bool(velocity)
        self.precision = precision

    def __call__(self, y):
        if self.precision == 'mixed':
            return self.engine.apply(y.to(torch.complex64), self.field, self.velocity,
                                     precision='complex64').to(torch.complex128)
        return self.engine.apply(y, self.field, self.velocity)


class FieldSchedule:
    """(t, y) -> H(field(t)) y of a B200Hamiltonian; ``step`` recognises it and uses
    the fused device Arnoldi."""

    def __init__(self, engine, field_at, velocity=True, precision='complex128'):
        self.engine = engine
        self.field_at = field_at
        self.velocity = bool(velocity)
        self.precision = precision

    def __call__(self, t, y):
        return self.at(t)(y)

    def at(self, t):
        return FieldOperator(self.engine, self.field_at(t), self.velocity, self.precision)


def _not_converged(maxdim, dt, err):
    return RuntimeError(f'GPU Arnoldi did not converge: dim={maxdim}, dt={dt}, estimate={err:.3e}')


@torch.no_grad()
def exponential_action(apply, x, dt, tol=1e-10, maxdim=48):
    """exp(-i dt H) x by Arnoldi (python/torch_backend.py:140-158)."""
    if x.dtype != torch.complex128 or x.device.type != 'cuda':
        raise ValueError('exponential_action needs a complex128 CUDA tensor')
    x = x.contiguous()
    ws = workspace(x.numel(), maxdim, x.device)
    stream = _stream(x.device)
    if isinstance(apply, FieldOperator):
        return _fused(apply, ws, x, dt, tol, maxdim, stream)
    beta = ct.c_double()
    check(LIB.he_krylov_start(ws.handle, ct.c_void_p(x.data_ptr()), ct.byref(beta), stream), 'he_krylov_start')
    if beta.value == 0:
        return x.clone(), {'dimension': 0, 'residual_estimate': 0.}
    done, m, err = ct.c_int(0), ct.c_int(0), ct.c_double(0.)
    for j in range(maxdim):
        v = apply(ws.vector(j))
        ws.vector(j + 1).copy_(v)
        check(LIB.he_krylov_orthogonalize(ws.handle, j, stream), 'he_krylov_orthogonalize')
        sync = (j >= 3 and ((j + 1) % 4 == 0 or j + 1 == maxdim)) or j + 1 == maxdim
        status = LIB.he_expv_check(ws.handle, j, maxdim, float(dt), float(tol), int(sync), ct.byref(done),
                                   ct.byref(m), ct.byref(err), stream)
        if status == HE_ERR_NOCONV:
            raise _not_converged(maxdim, dt, err.value)
        check(status, 'he_expv_check')
        if sync and done.value:
            y = torch.empty_like(x)
            check(LIB.he_krylov_combine(ws.handle, m.value, ct.c_void_p(y.data_ptr()), stream), 'he_krylov_combine')
            return y, {'dimension': m.value, 'residual_estimate': float(err.value)}
    raise _not_converged(maxdim, dt, err.value)


def _fused(op, ws, x, dt, tol, maxdim, stream):
    y = torch.empty_like(x)
    dim, err = ct.c_int(0), ct.c_double(0.)
    fn = LIB.he_expv_mixed if op.precision == 'mixed' else LIB.he_expv
    status = fn(ws.handle, op.engine.op.handle, ct.c_void_p(x.data_ptr()), ct.c_void_p(y.data_ptr()),
                         ptr(op.field), int(op.velocity), float(dt), float(tol), int(maxdim), ct.byref(dim),
                         ct.byref(err), stream)
    if status == HE_ERR_NOCONV:
        op.engine.apply_count += int(maxdim)   # the attempt ran to maxdim
        raise _not_converged(maxdim, dt, err.value)
    check(status, 'he_expv')
    op.engine.apply_count += dim.value
    return y, {'dimension': dim.value, 'residual_estimate': float(err.value)}


@torch.no_grad()
def field_derivative_action(engine, x, field, direction, dt, tol=1e-10, maxdim=48):
    """exp(-i dt B) x for B = [[H(field), direction . d], [0, H(field)]] on x = [u; w], a
    complex128 device vector of 2 engine.size values (length gauge, he_expv_field_derivative):
    the lower half of the result is exp(-i dt H) w, the upper half exp(-i dt H) u + L w with L
    the derivative of exp(-i dt H(field)) along the field direction.  One fused Arnoldi on the
    block operator (a two-instance apply and one dipole pass per Krylov vector)."""
    if x.dtype != torch.complex128 or x.device.type != 'cuda' or x.numel() != 2 * engine.size:
        raise ValueError('field_derivative_action needs a complex128 CUDA vector of 2 engine.size values')
    x = x.contiguous()
    ws = workspace(x.numel(), maxdim, x.device)
    y = torch.empty_like(x)
    f = np.ascontiguousarray(field, dtype=np.float64)
    d = np.ascontiguousarray(direction, dtype=np.float64)
    dim, err = ct.c_int(0), ct.c_double(0.)
    status = LIB.he_expv_field_derivative(ws.handle, engine.op.handle, ct.c_void_p(x.data_ptr()),
                                          ct.c_void_p(y.data_ptr()), ptr(f), ptr(d), float(dt), float(tol),
                                          int(maxdim), ct.byref(dim), ct.byref(err), _stream(x.device))
    if status == HE_ERR_NOCONV:
        raise _not_converged(maxdim, dt, err.value)
    check(status, 'he_expv_field_derivative')
    engine.apply_count += 2 * dim.value
    return y, {'dimension': dim.value, 'residual_estimate': float(err.value)}


class BatchedWorkspace:
    """Krylov workspace for ``count`` instances advanced together (he_krylov_create_batched)."""

    def __init__(self, n, maxdim, count, device):
        self.n, self.maxdim, self.count, self.device = int(n), int(maxdim), int(count), torch.device(device)
        handle = ct.c_void_p()
        with torch.cuda.device(self.device):
            check(LIB.he_krylov_create_batched(ct.byref(handle), self.n, self.maxdim, self.count),
                  'he_krylov_create_batched')
        self.handle = handle
        if _GRAPHS[0]:
            check(LIB.he_krylov_set_graphs(handle, 1), 'he_krylov_set_graphs')

    def __del__(self):
        handle = getattr(self, 'handle', None)
        if handle is not None and handle.value:
            LIB.he_krylov_destroy(handle)
            self.handle = None


_BATCHED = {}


def batched_workspace(n, maxdim, count, device):
    device = torch.device(device)
    key = (device, int(n), int(count), torch.cuda.current_stream(device).cuda_stream)
    ws = _BATCHED.get(key)
    if ws is None or ws.maxdim < maxdim:
        ws = BatchedWorkspace(n, max(maxdim, ws.maxdim if ws else 0), count, device)
        _BATCHED[key] = ws
    return ws


@torch.no_grad()
def step_batched(engine, fields_at, x, t, dt, tol=1e-10, maxdim=48, velocity=False, precision='complex128', depth=0):
    """One midpoint Arnoldi step of ``count`` instances sharing ``engine``: x is
    (count, size) complex128, ``fields_at(t)`` returns the (count, 3) fields.  The batch
    runs as one device Arnoldi (he_expv_batched).  Instances that do not converge at dt
    are redone together with the reference's recursive halving (two half steps, depth
    <= 8, tolerance halved), so every instance gets the result of stepping it by itself
    with :func:`step`.  Returns (y, info) with per-instance dimensions."""
    count = x.shape[0]
    if x.dtype != torch.complex128 or not x.is_contiguous() or x.numel() != count * engine.size:
        raise ValueError('batch must be a contiguous complex128 (count, size) tensor')
    ws = batched_workspace(engine.size, maxdim, count, x.device)
    fields = np.ascontiguousarray(fields_at(t + dt / 2), dtype=np.float64).reshape(count, 3)
    y = torch.empty_like(x)
    dims = np.zeros(count, np.int32)
    est = np.zeros(count)
    conv = np.zeros(count, np.int32)
    code = {'complex128': 0, 'mixed': 1}[precision]
    status = LIB.he_expv_batched(ws.handle, engine.op.handle, ct.c_void_p(x.data_ptr()), ct.c_void_p(y.data_ptr()),
                                 ptr(fields), int(bool(velocity)), float(dt), float(tol), int(maxdim), code,
                                 ptr(dims), ptr(est), ptr(conv), _stream(x.device))
    if status != HE_ERR_NOCONV:
        check(status, 'he_expv_batched')
    engine.apply_count += int(dims.sum())
    info = {'dimension': dims.copy(), 'residual_estimate': est.copy(), 'subdivided': np.zeros(count, bool)}
    failed = np.flatnonzero(conv == 0)
    if len(failed):
        if depth >= 8:
            raise _not_converged(maxdim, dt, float(est[failed].max()))
        sub = lambda tt: np.asarray(fields_at(tt)).reshape(count, 3)[failed]
        xs = x[torch.as_tensor(failed, device=x.device)].contiguous()
        ys, a = step_batched(engine, sub, xs, t, dt / 2, tol / 2, maxdim, velocity, precision, depth + 1)
        ys, b = step_batched(engine, sub, ys, t + dt / 2, dt / 2, tol / 2, maxdim, velocity, precision, depth + 1)
        y[torch.as_tensor(failed, device=x.device)] = ys
        info['dimension'][failed] = np.maximum(a['dimension'], b['dimension'])
        info['residual_estimate'][failed] = a['residual_estimate'] + b['residual_estimate']
        info['subdivided'][failed] = True
    return y, info


def step(apply_at, x, t, dt, tol=1e-10, maxdim=48, depth=0):
    """Midpoint exponential step with recursive halving (python/torch_backend.py:160-167).
    info['path'] lists the accepted exponentials in order as (t, dt, tol, dimension)."""
    try:
        if isinstance(apply_at, FieldSchedule):
            operator = apply_at.at(t + dt / 2)
        else:
            operator = lambda y: apply_at(t + dt / 2, y)
        y, info = exponential_action(operator, x, dt, tol, maxdim)
        info['path'] = [(t, dt, tol, info['dimension'])]
        return y, info
    except RuntimeError as error:
        if 'Arnoldi did not converge' not in str(error) or depth >= 8:
            raise
        y, a = step(apply_at, x, t, dt / 2, tol / 2, maxdim, depth + 1)
        y, b = step(apply_at, y, t + dt / 2, dt / 2, tol / 2, maxdim, depth + 1)
        return y, {'dimension': max(a['dimension'], b['dimension']),
                   'residual_estimate': a['residual_estimate'] + b['residual_estimate'], 'subdivided': True,
                   'path': a['path'] + b['path']}


__all__ = ['TorchHamiltonian', 'B200Hamiltonian', 'exponential_action', 'step', 'step_batched', 'FieldOperator',
           'FieldSchedule', 'HeliumError']
