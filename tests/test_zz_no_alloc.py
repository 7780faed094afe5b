"""he_vec_norms_noalloc: batched norms whose scratch is a fixed device array, for
callers that cannot let a library call allocate device memory (a process whose device
memory belongs to a pool allocator, a latency-critical loop that must not stall on the
allocator, a runtime that forbids allocations outside its own allocator).

Checked through the C-ABI against the allocating entry point he_vec_residual_norm, on two
calls in a row (the second call reuses the shared scratch left by the first), at the
tolerance the other norm/Krylov tests use (1e-14 relative); the device's free memory
(cudaMemGetInfo) is the same before and after a call once the array exists, with the
default lazy module loading and with CUDA_MODULE_LOADING=EAGER (in a child process).  This
file is collected last so that a run stopping at the first failure has already run every
other test.
"""
import ctypes as ct
import os
import subprocess
import sys
from pathlib import Path

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


def test_noalloc_call_leaves_device_free_memory_unchanged():
    """After the first call on the device (which, under lazy module loading, is when the
    driver allocates the static array), further calls allocate nothing."""
    from laqphysics_b200._lib import LIB
    n, count = 100_003, 16
    x = torch.randn((count, n), dtype=torch.complex128, device=DEVICE)
    assert _noalloc_norms(LIB, x, count, n, n)[0] == 0
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info(DEVICE)
    for _ in range(3):
        status, norms = _noalloc_norms(LIB, x, count, n, n)
        assert status == 0
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info(DEVICE)
    assert free_after == free_before
    np.testing.assert_allclose(norms, torch.linalg.vector_norm(x, dim=1).cpu().numpy(), rtol=1e-12)


def test_noalloc_under_eager_module_loading():
    """The same checks in a fresh process with CUDA_MODULE_LOADING=EAGER (the array is then
    allocated with the context, before the first call)."""
    here = Path(__file__).resolve()
    env = dict(os.environ, CUDA_MODULE_LOADING='EAGER')
    code = ('import sys; sys.path.insert(0, %r); import test_zz_no_alloc as t; '
            't.test_noalloc_norms_match_allocating_entry_point_on_two_calls(); '
            't.test_noalloc_call_leaves_device_free_memory_unchanged(); print("ok")') % str(here.parent)
    out = subprocess.run([sys.executable, '-c', code], env=env, cwd=str(here.parents[1]), capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0 and out.stdout.strip().endswith('ok'), out.stdout + out.stderr
