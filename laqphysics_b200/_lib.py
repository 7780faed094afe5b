"""ctypes binding of libhelium_b200.so (the C-ABI declared in include/helium_b200.h).

The library is required: importing this module without it raises, so no code path
can silently run without the CUDA kernels.  Build it with
``python -m laqphysics_b200.build``.
"""
import ctypes as ct
import os
from pathlib import Path

LIBRARY = Path(os.environ.get('HELIUM_B200_LIBRARY', Path(__file__).resolve().parent / '_lib' / 'libhelium_b200.so'))
if not LIBRARY.exists():
    raise ImportError(f'{LIBRARY} is missing: build it with `python -m laqphysics_b200.build`')
LIB = ct.CDLL(str(LIBRARY))

HE_OK, HE_ERR_ARG, HE_ERR_SHAPE, HE_ERR_CUDA, HE_ERR_NOCONV, HE_ERR_UNSUPPORTED, HE_ERR_DEVICE = range(7)
HE_C128, HE_C64 = 0, 1

P = ct.c_void_p
I = ct.c_int
D = ct.c_double

# Every exported symbol and its argument types: (name, restype, argtypes).
SIGNATURES = {
    'tensor_apply': (None, [I, I, I, P, P, P, P, I, P, P, P, P, P, I, P, P, P, P, P, P, P, I, P, P]),
    'he_last_status': (I, []),
    'he_last_error': (ct.c_char_p, []),
    'he_version': (I, []),
    'he_binary_version': (I, [ct.POINTER(I)]),
    'he_create': (I, [ct.POINTER(P), I, I, I, P, P, P, P, P, P, I, P, P, P, P, P, I, I, P, P, P, P, P, P, I]),
    'he_destroy': (I, [P]),
    'he_info': (I, [P, ct.POINTER(ct.c_longlong), I]),
    'he_apply': (I, [P, P, P, P, I, I, P]),
    'he_apply_batched': (I, [P, I, P, P, P, I, I, P]),
    'he_apply_shifted': (I, [P, P, P, P, I, D, D, D, I, P]),
    'he_diagonal': (I, [P, P, P]),
    'he_flux': (I, [P, P, P, I, I, I, P, P, P, P]),
    'he_krylov_create': (I, [ct.POINTER(P), ct.c_longlong, I, I]),
    'he_krylov_destroy': (I, [P]),
    'he_krylov_vector': (I, [P, I, I, ct.POINTER(P)]),
    'he_krylov_start': (I, [P, P, ct.POINTER(D), P]),
    'he_krylov_orthogonalize': (I, [P, I, P]),
    'he_expv_check': (I, [P, I, I, D, D, I, ct.POINTER(I), ct.POINTER(I), ct.POINTER(D), P]),
    'he_krylov_combine': (I, [P, I, P, P]),
    'he_expv': (I, [P, P, P, P, P, I, D, D, I, ct.POINTER(I), ct.POINTER(D), P]),
    'he_expv_mixed': (I, [P, P, P, P, P, I, D, D, I, ct.POINTER(I), ct.POINTER(D), P]),
    'he_krylov_create_batched': (I, [ct.POINTER(P), ct.c_longlong, I, I]),
    'he_expv_batched': (I, [P, P, P, P, P, I, D, D, I, I, P, P, P, P]),
    'he_set_path': (I, [P, I]),
    'he_device_status': (I, [P]),
    'he_set_mix': (I, [P, I]),
    'he_mix_status': (I, [P]),
    'he_set_mix_blocks': (I, [P, I, I]),
    'he_set_band_stages': (I, [P, I, I]),
    'he_fp64_peak': (I, [I, I, ct.POINTER(ct.c_double), P]),
    'he_set_mixed_gauge': (I, [P, P, P, P, P, P, I, P, P, P, P]),
    'he_apply_mixed_terms': (I, [P, P, P, P, P]),
    'he_apply_dipole': (I, [P, P, P, P, P]),
    'he_ionic_create': (I, [ct.POINTER(P), I, I, I, ct.c_longlong, P, P, P]),
    'he_ionic_set_preconditioner': (I, [P, I, I, P, P, P]),
    'he_ionic_apply': (I, [P, P, I, P, P, D, D, D, I, P]),
    'he_ionic_precondition': (I, [P, P, P, D, D, D, P]),
    'he_ionic_destroy': (I, [P]),
    'he_plan_mix_source': (ct.c_longlong, [P, I, ct.c_char_p, ct.c_longlong]),
    'he_nvrtc_check': (I, [ct.c_char_p, ct.c_char_p, ct.c_longlong]),
    'he_plan_mix_program': (ct.c_longlong, [P, ct.c_char_p, ct.c_longlong]),
    'he_vec_axpby': (I, [ct.c_longlong, D, D, P, D, D, P, P, P]),
    'he_vec_residual_norm': (I, [ct.c_longlong, P, P, P, ct.POINTER(D), P]),
    'he_vec_jacobi': (I, [ct.c_longlong, P, D, D, D, P, P, P]),
    'he_krylov_scale': (I, [P, I, I, D, P]),
    'he_krylov_normalize': (I, [P, I, P]),
    'he_krylov_set_graphs': (I, [P, I]),
    'he_krylov_capture_fallbacks': (I, [P, ct.POINTER(I), ct.POINTER(I)]),
    'he_expv_field_derivative': (I, [P, P, P, P, P, P, D, D, I, ct.POINTER(I), ct.POINTER(D), P]),
    'he_krylov_hessenberg': (I, [P, I, I, P, P]),
    'he_krylov_reset': (I, [P, P]),
    'he_krylov_combine_coef': (I, [P, I, I, P, P, I, P]),
    'he_separable_create': (I, [ct.POINTER(P), I, I, I, P, P, P, P, P, I]),
    'he_separable_destroy': (I, [P]),
    'he_separable_apply': (I, [P, P, P, D, D, D, P]),
    'he_separable_set_passes': (I, [P, I]),
    'he_separable_set_tile': (I, [P, I]),
    'he_gmres_shifted': (I, [P, P, P, P, P, P, P, D, D, D, D, D, I, I, I, ct.POINTER(I), ct.POINTER(D), P]),
    'he_cf4_step': (I, [P, P, P, P, P, P, P, D, D, D, D, I, I, ct.POINTER(I), ct.POINTER(D), P]),
    'he_cf4_coefficients': (I, [P, D, D, D, P]),
    'he_gmres_segment_hint': (I, [P, ct.POINTER(I), ct.POINTER(ct.c_longlong)]),
    'he_separable_status': (I, [P]),
    'he_surface_contract': (I, [ct.c_longlong, I, I, I, I, P, P, ct.c_longlong, ct.c_longlong, ct.c_longlong,
                                P, P, P, P, P, P, P, P]),
    'he_volkov_add': (I, [I, I, I, I, I, P, P, P, P, P, P, D, P, D, D, I, P, P, P]),
    'he_sample_create': (I, [P, P, I, I, I, P, P, I, I, I, P, P, P, P, P, P, I, I, P, P, P, P, P]),
    'he_sample_record': (I, [P, P, P, P, D, P, D, D, I, P, P, P, P, P]),
    'he_sample_grid': (I, [P]),
    'he_sample_set_wait_extra': (I, [P, ct.c_uint]),
    'he_sample_status': (I, [P]),
    'he_sample_destroy': (I, [P]),
    'he_vec_norms_noalloc': (I, [ct.c_longlong, I, P, ct.c_longlong, P, P]),
    'he_diagnostics': (I, [P, P, P, P, P, P, ct.POINTER(D), P]),
    'he_plan_build': (P, [I, I, P, P, P, I, P, P, P, P, I, I, P, P, P, P]),
    'he_plan_free': (None, [P]),
    'he_plan_array': (ct.c_longlong, [P, I, P]),
}

for _name, (_res, _args) in SIGNATURES.items():
    _fn = getattr(LIB, _name)
    _fn.restype = _res
    _fn.argtypes = _args


class HeliumError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status, message):
        super().__init__(f'{message} (status {status})')
        self.status = status


def check(status, what=''):
    if status != HE_OK:
        message = LIB.he_last_error().decode(errors='replace')
        raise HeliumError(status, f'{what}: {message}' if what else message)
    return status


def ptr(array):
    """Address of a numpy array's data as a ctypes void pointer."""
    return ct.c_void_p(array.ctypes.data)
