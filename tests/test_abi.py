"""The C-ABI library loads, exports every symbol include/*.h declares, and validates
its inputs on the host (no GPU needed for any of these checks)."""
import ctypes as ct
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import REPO, Tables, golden

HEADERS = sorted((REPO / 'include').glob('*.h'))


def declared_functions():
    names = set()
    for header in HEADERS:
        text = re.sub(r'/\*.*?\*/', '', header.read_text(), flags=re.S)
        for match in re.finditer(r'^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(', text, flags=re.M):
            if not match.group(0).lstrip().startswith(('typedef', 'enum', '#')):
                names.add(match.group(1))
    return sorted(names)


def test_header_declares_the_drop_in_symbol():
    names = declared_functions()
    assert 'tensor_apply' in names and 'he_apply' in names and len(names) >= 10


def test_library_exports_every_declared_symbol():
    from laqphysics_b200 import _lib
    for name in declared_functions():
        assert hasattr(_lib.LIB, name), name
        assert name in _lib.SIGNATURES, f'{name} has no ctypes signature'


def test_library_is_built_for_sm100a_only():
    """The build compiles every CUDA source for sm_100a and nothing else (the architecture
    a kernel actually ran with is checked on the GPU through cudaFuncGetAttributes)."""
    from laqphysics_b200 import build
    assert build.ARCH == ['-gencode', 'arch=compute_100a,code=sm_100a']
    assert not any('arch=' in flag or 'code=' in flag for flag in build.FLAGS)


def _create(h, **overrides):
    from laqphysics_b200 import _lib
    from laqphysics_b200.engine import _host_tables
    t = _host_tables(h)
    t.update(overrides)
    p = lambda a: _lib.ptr(a) if a is not None else None
    handle = ct.c_void_p()
    status = _lib.LIB.he_create(ct.byref(handle), t.get('n', h.n), h.nc, len(t['tv']), p(t['ptr']), p(t['col']),
                                p(t['tv']), p(t['diag']), p(t['d1']), p(t['d2']), len(t['vc']), p(t['vptr']),
                                p(t['vc']), p(t['vl']), p(t['vcoef']), p(t['rad']), t['nlam'], len(t['dc']),
                                p(t['dptr']), p(t['dc']), p(t['de']), p(t['dcoef']), p(t['ldiff']), p(t['r']), 0)
    return status, _lib.LIB.he_last_error().decode()


def test_create_rejects_out_of_range_kinetic_column():
    from laqphysics_b200 import _lib
    h = Tables(golden('apply_ecs'))
    col = h.col.copy()
    col[3] = h.n + 5
    status, message = _create(h, col=col)
    assert status == _lib.HE_ERR_SHAPE and 'kinetic' in message


def test_create_rejects_multipole_outside_rad_table():
    from laqphysics_b200 import _lib
    h = Tables(golden('apply_ecs'))
    vl = h.vl.copy()
    vl[0] = 99
    status, message = _create(h, vl=vl)
    assert status == _lib.HE_ERR_SHAPE and 'multipole' in message


def test_create_rejects_bad_dipole_electron_and_missing_diagonal():
    from laqphysics_b200 import _lib
    h = Tables(golden('apply_ecs'))
    de = h.de.copy()
    de[0] = 3
    assert _create(h, de=de)[0] == _lib.HE_ERR_SHAPE
    assert _create(h, diag=None)[0] == _lib.HE_ERR_ARG


def test_apply_rejects_null_handle_and_bad_precision():
    from laqphysics_b200 import _lib
    f = np.zeros(3)
    assert _lib.LIB.he_apply(None, None, None, _lib.ptr(f), 0, 0, None) == _lib.HE_ERR_ARG


def test_native_tensor_apply_validates_field_shape():
    from laqphysics_b200.native import tensor_apply
    h = Tables(golden('apply_ecs'))
    with pytest.raises(ValueError, match='three Cartesian'):
        tensor_apply(h, np.zeros(h.size, complex), field=(0., 1.))


def test_step_and_sample_entries_reject_bad_arguments_on_the_host():
    """he_cf4_step, he_gmres_shifted and the surface-sample entries check their pointers
    and sizes before any device work: HE_ERR_ARG with a message, no CUDA call needed."""
    from laqphysics_b200._lib import HE_ERR_ARG, LIB
    i, d = ct.c_int(), ct.c_double()
    fields = np.zeros(6)
    assert LIB.he_cf4_step(None, None, None, None, None, None, fields.ctypes.data, .05, 0., 1., 1e-10, 16, 10,
                           ct.byref(i), ct.byref(d), None) == HE_ERR_ARG
    assert b'CF4' in LIB.he_last_error()
    assert LIB.he_gmres_shifted(None, None, None, None, None, None, fields.ctypes.data, .01, 0., 0., 0., 1e-10, 16, 10,
                                0, ct.byref(i), ct.byref(d), None) == HE_ERR_ARG
    assert LIB.he_sample_create(ct.byref(ct.c_void_p()), None, 1, 0, 1, None, None, 1, 1, 1, None, None, None, None,
                                None, None, 1, 1, None, None, None, None, None) == HE_ERR_ARG
    assert LIB.he_sample_record(None, None, None, None, 0., None, 0., 0., 1, None, None, None, None, None) == HE_ERR_ARG
    assert LIB.he_sample_status(None) == HE_ERR_ARG
    assert LIB.he_sample_set_wait_extra(None, 1) == HE_ERR_ARG
    assert LIB.he_sample_grid(None) == 0
    assert LIB.he_gmres_segment_hint(None, ct.byref(i), None) == HE_ERR_ARG


@pytest.mark.parametrize('a2, e_ref', [(1., -2.9), (.5, 0.), (1., .37)])
def test_cf4_step_host_arithmetic_matches_the_python_step(a2, e_ref):
    """he_cf4_coefficients (the arithmetic he_cf4_step runs on the host) against the
    formulas of implicit.cf4_step / pade_step (python/implicit.py:91-109, :76-89): effective
    fields, preconditioner shifts, phase angles and the two Pade alphas."""
    from laqphysics_b200._lib import HE_OK, LIB
    from laqphysics_b200.implicit import A1, A2, C1, C2, SQRT3
    rng = np.random.default_rng(11)
    fields = np.ascontiguousarray(rng.normal(scale=.05, size=(2, 3)))
    dt = .05
    out = np.zeros(14)
    assert LIB.he_cf4_coefficients(fields.ctypes.data, dt, e_ref, a2, out.ctypes.data) == HE_OK
    for e, w in enumerate(((A2, A1), (A1, A2))):
        effective = 2 * np.einsum('a,aj->j', w, fields)
        correction = a2 * (np.dot(w, np.sum(fields ** 2, axis=1)) - .5 * np.dot(effective, effective))
        shift = a2 * sum(float(a) ** 2 for a in effective) - e_ref
        np.testing.assert_allclose(out[5 * e:5 * e + 3], effective, rtol=1e-15, atol=1e-18)
        np.testing.assert_allclose(out[5 * e + 3], shift, rtol=1e-14, atol=1e-16)
        np.testing.assert_allclose(out[5 * e + 4], -dt * (correction + e_ref / 2), rtol=1e-13, atol=1e-17)
    for r, root in enumerate((3 + 1j * SQRT3, 3 - 1j * SQRT3)):
        alpha = (dt / 2) / root
        np.testing.assert_allclose(out[10 + 2 * r] + 1j * out[11 + 2 * r], alpha, rtol=1e-15)
    assert C1 < C2
