"""he_vec_norms_noalloc: batched norms whose scratch is a fixed device array, for
callers that cannot let a library call allocate device memory (a process whose device
memory belongs to a pool allocator, a latency-critical loop that must not stall on the
allocator, a runtime that forbids allocations outside its own allocator).

Checked through the C-ABI against the allocating entry point he_vec_residual_norm, on two
calls in a row (the second call reuses the shared scratch left by the first), at the
tolerance the other norm/Krylov tests use (1e-14 relative).  This file is collected last
so that a run stopping at the first failure has already run every other test.
"""
import ctypes as ct

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'


def _stream():
    return ct.c_void_p(torch.cuda.current_stream(DEVICE).cuda_stream)


def _existing_norm(lib, v):
    value = ct.c_double()
    assert lib.he_vec_residual_norm(v.numel(), ct.c_void_p(v.data_ptr()), None, None, ct.byref(value), _stream()) == 0
    return value.value


def _noalloc_norms(lib, x, count, ld, n):
    norms = np.zeros(count)
    status = lib.he_vec_norms_noalloc(n, count, ct.c_void_p(x.data_ptr()), ld, norms.ctypes.data, _stream())
    return status, norms


def test_noalloc_norms_match_allocating_entry_point_on_two_calls():
    from laqphysics_b200._lib import LIB
    n = 300_007                         # not a multiple of the block size
    rng = np.random.default_rng(2024)
    for call, count in enumerate((7, 64)):
        ld = n + 3
        host = (rng.normal(size=(count, ld)) + 1j * rng.normal(size=(count, ld))) * (call + 1)
        x = torch.as_tensor(host, device=DEVICE)
        status, norms = _noalloc_norms(LIB, x, count, ld, n)
        assert status == 0, LIB.he_last_error().decode()
        expected = np.array([_existing_norm(LIB, x[v, :n].contiguous()) for v in range(count)])
        np.testing.assert_allclose(norms, expected, rtol=1e-14, atol=0)
        np.testing.assert_allclose(norms, np.linalg.norm(host[:, :n], axis=1), rtol=1e-12)


def test_noalloc_norms_reject_batches_beyond_the_scratch():
    from laqphysics_b200._lib import HE_ERR_ARG, LIB
    x = torch.zeros((65, 16), dtype=torch.complex128, device=DEVICE)
    status, _ = _noalloc_norms(LIB, x, 65, 16, 16)
    assert status == HE_ERR_ARG
    assert 'count must be between 1 and 64' in LIB.he_last_error().decode()
