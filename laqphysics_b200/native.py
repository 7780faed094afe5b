"""Drop-in for the reference's ``native.tensor_apply`` (python/native.py:24-38).

Same call, same marshalling of the table arrays and the same Fortran-ordered
complex128 result, but the work runs on the GPU through this package's C-ABI
symbol ``tensor_apply`` (include/helium_b200.h).  A failure raises instead of being
silent: the C symbol keeps the reference's void signature and reports through
``he_last_status`` / ``he_last_error``.
"""
import numpy as np

from ._lib import LIB, check, ptr

TABLES_INT = ('ptr', 'col', 'vptr', 'vc', 'vl', 'dptr', 'dc', 'de')
TABLES_COMPLEX = ('tv', 'diag', 'vcoef', 'rad', 'dcoef', 'r')


def _table(h, name):
    a = getattr(h, name)
    if name in TABLES_INT:
        want = np.int32
    elif name == 'ldiff':
        want = np.float64
    else:
        want = np.complex128
    if a.dtype != want or not (a.flags.f_contiguous or a.ndim <= 1 and a.flags.c_contiguous):
        raise ValueError(f'table {name} must be a contiguous {np.dtype(want).name} array in Fortran order')
    return a


def tensor_apply(h, psi, field=(0., 0., 0.), velocity=False):
    z = np.asfortranarray(np.asarray(psi).reshape(h.shape, order='F'), dtype=np.complex128)
    out = np.empty_like(z, order='F')
    f = np.ascontiguousarray(field, dtype=np.float64)
    if f.shape != (3,):
        raise ValueError('field must have three Cartesian components')
    t = {name: _table(h, name) for name in TABLES_INT + TABLES_COMPLEX + ('ldiff',)}
    LIB.tensor_apply(h.n, h.nc, len(t['tv']), ptr(t['ptr']), ptr(t['col']), ptr(t['tv']), ptr(t['diag']),
                     len(t['vc']), ptr(t['vptr']), ptr(t['vc']), ptr(t['vl']), ptr(t['vcoef']), ptr(t['rad']),
                     len(t['dc']), ptr(t['dptr']), ptr(t['dc']), ptr(t['de']), ptr(t['dcoef']), ptr(t['ldiff']),
                     ptr(t['r']), ptr(f), int(bool(velocity)), ptr(z), ptr(out))
    check(LIB.he_last_status(), 'tensor_apply')
    return out.ravel(order='F')
