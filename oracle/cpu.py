"""ORACLE (test infrastructure only): ctypes access to oracle/_build/libhelium_oracle.so,
the C/OpenMP restatement of the reference's tensor_apply (src/kernels.f90:119-176).

Marshalling is the reference's python/native.py:24-38: Fortran-ordered complex128
tables and state, zero-based int32 indices, `out` preallocated here.
"""
import ctypes as ct
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / '_build' / 'libhelium_oracle.so'
_lib = None


def build():
    subprocess.run(['make', '-s', '-C', str(HERE)], check=True)
    return LIBRARY


def lib():
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            build()
        _lib = ct.CDLL(str(LIBRARY))
        _lib.tensor_apply.restype = None
        _lib.tensor_apply_channels.restype = None
        _lib.oracle_max_threads.restype = ct.c_int
    return _lib


def _p(a):
    return ct.c_void_p(a.ctypes.data)


def threads():
    return lib().oracle_max_threads()


def host_tables(h):
    """The table arrays in the dtypes/orders the C ABI expects (python/native.py:31-37)."""
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    cf = lambda a: np.asfortranarray(a, dtype=np.complex128)
    t = {k: i32(getattr(h, k)) for k in ('ptr', 'col', 'vptr', 'vc', 'vl', 'dptr', 'dc', 'de')}
    for k in ('tv', 'diag', 'vcoef', 'rad', 'dcoef', 'r'):
        t[k] = cf(getattr(h, k))
    t['ldiff'] = np.ascontiguousarray(h.ldiff, dtype=np.float64)
    return t


def tensor_apply(h, psi, field=(0., 0., 0.), velocity=False, channels=None, tables=None):
    """Reference H·psi on the host CPU (OpenMP threads from OMP_NUM_THREADS).

    ``channels=(c0, c1)`` computes only output channels [c0, c1) (other outputs stay
    uninitialised); ``tables`` reuses a ``host_tables(h)`` result."""
    z = np.asfortranarray(np.asarray(psi).reshape(h.shape, order='F'), dtype=np.complex128)
    out = np.empty_like(z, order='F')
    f = np.ascontiguousarray(field, dtype=np.float64)
    if f.shape != (3,):
        raise ValueError('field must have three Cartesian components')
    t = tables if tables is not None else host_tables(h)
    c0, c1 = (0, h.nc) if channels is None else channels
    lib().tensor_apply_channels(
        ct.c_int(h.n), ct.c_int(h.nc), ct.c_int(len(t['tv'])), _p(t['ptr']), _p(t['col']), _p(t['tv']), _p(t['diag']),
        ct.c_int(len(t['vc'])), _p(t['vptr']), _p(t['vc']), _p(t['vl']), _p(t['vcoef']), _p(t['rad']),
        ct.c_int(len(t['dc'])), _p(t['dptr']), _p(t['dc']), _p(t['de']), _p(t['dcoef']), _p(t['ldiff']), _p(t['r']),
        _p(f), ct.c_int(int(bool(velocity))), _p(z), _p(out), ct.c_int(c0), ct.c_int(c1))
    return out.ravel(order='F')
