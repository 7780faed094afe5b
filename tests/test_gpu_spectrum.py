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


def test_device_tsurff_run_matches_the_reference_driver_run():
    """The whole run against the reference's own production driver on the same case
    (tests/golden/tsurff_run.npz: python/run3d.py with the Torch backend on the CPU and online
    spectrum storage, OnlineSurface + VolkovAccumulator): the same 365-step time grid
    (T / ceil(T / dt)), the reference's ground state as the start, Krylov dimension 16 and
    tolerance 1e-10.  This pins the composition (frame indexing, channel-function frame
    alignment, the trapezoid at the first and last samples), not only the pieces.
    Bounds (relative L2 against the reference run): complex128 spectrum and amplitudes 1e-9,
    final state 1e-10; mixed precision spectrum 1e-6 (the stated mixed-precision target)."""
    import json
    from conftest import golden
    from laqphysics_b200.tsurff_run import SMALL_CASE, build_case, run
    g = golden('tsurff_run')
    config = json.loads(str(g['config']))
    dt = float(g['dt'])
    engine, contractor, psi0, avec, steps, chi = build_case(SMALL_CASE, DEVICE, dt, config['post_time'], g['ground'])
    assert steps == int(g['nsteps'])
    kw = dict(tol=config['krylov_tolerance'], maxdim=config['krylov_dimension'])
    acc64, psi64, _ = run(engine, contractor, SMALL_CASE, psi0, avec, dt, steps, chi, 'complex128', **kw)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    pes, total = acc64.spectrum()
    np.testing.assert_allclose(acc64.energy, g['energy'], rtol=1e-15)
    assert rel(acc64.amplitude.cpu().numpy(), g['amplitudes']) <= 1e-9
    assert rel(pes, g['pes']) <= 1e-9
    assert rel(total, g['angle_integrated']) <= 1e-9
    assert rel(engine.host(psi64), g['psi']) <= 1e-10
    acc32, psi32, _ = run(engine, contractor, SMALL_CASE, psi0, avec, dt, steps, chi, 'mixed', **kw)
    pes32, _ = acc32.spectrum()
    assert rel(pes32, g['pes']) <= 1e-6
