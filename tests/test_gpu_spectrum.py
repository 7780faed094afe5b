"""Mixed precision against complex128 on a whole channel-resolved tSURFF run: velocity-
gauge Arnoldi propagation from the ground state through a short pulse, a surface sample
every step, He+ (n <= 2) channel spectra.  The mixed run applies H·psi in complex64 inside
the complex128 Krylov; everything on the surface stays complex128.

Stated tolerances (mixed vs complex128): photoelectron spectrum relative L2 error <= 1e-6
(the mixed-precision target), final-state relative L2 error <= 2e-6, norm difference
<= 1e-8."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'


def test_mixed_precision_tsurff_spectrum_against_complex128():
    from laqphysics_b200.tsurff_run import SMALL_CASE, build_case, run, spectrum_error
    dt = .02
    engine, contractor, psi0, avec, steps, chi = build_case(SMALL_CASE, DEVICE, dt)
    acc64, psi64, _ = run(engine, contractor, SMALL_CASE, psi0, avec, dt, steps, chi, 'complex128')
    acc32, psi32, _ = run(engine, contractor, SMALL_CASE, psi0, avec, dt, steps, chi, 'mixed')
    rel, per_label = spectrum_error(acc32, acc64)
    pes, _ = acc64.spectrum()
    assert np.isfinite(pes).all() and pes.max() > 0
    assert rel <= 1e-6, rel
    state = float(torch.linalg.vector_norm(psi32 - psi64) / torch.linalg.vector_norm(psi64))
    assert state <= 2e-6, state
    assert abs(float(torch.linalg.vector_norm(psi32)) - float(torch.linalg.vector_norm(psi64))) <= 1e-8
