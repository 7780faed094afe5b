"""GPU parity of online tSURFF: the device ionic contraction and the FP64 Volkov
trapezoid accumulator against the reference's OnlineSurface run (golden fixture
'volkov': python/streaming_surface.py:39-64 + python/surface_contract.py:41-56 on the
reference test configuration tests/test_streaming_surface.py:10-20, linear coupled
variant).  Tolerance: the reference's own GPU-vs-numpy accumulator bound, 3e-12
(tests/test_streaming_surface.py:132)."""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'

CONFIG = {'radial': {'edges': [0, 1, 2, 4, 6, 8], 'order': 3, 'tail': 6, 'ecs_angle': .3},
          'lmax': 1, 'M': 0, 'total_Lmax': 2, 'cutoff_radii': [1, 2], 'surface': 5.,
          'pulses': [{'pulse': {'omega': 5., 'cycles': 2, 'field': .15}, 'polarization': 'z'}],
          'ionic_channels': [[1, 0, 0], [2, 0, 0], [2, 1, 0]],
          'spectrum_energy': [.2, 1.2, 7], 'spectrum': {'theta_points': 4, 'phi_points': 1}}


def _setup(config=CONFIG):
    from laqphysics_b200.pulses import Pulse
    from laqphysics_b200.surface3d import Ionic
    from laqphysics_b200.surface_contract import SurfaceContractor
    from laqphysics_b200.workloads import coupled
    rc = config['radial']
    h = coupled(rc['edges'], rc['order'], config['lmax'], config['total_Lmax'], ecs_angle=rc['ecs_angle'],
                tail=rc['tail'], cutoff_radii=tuple(config['cutoff_radii']))
    base = h.uncoupled
    base.prepare_surface(config['surface'])
    h.prepare_surface(config['surface'])
    labels = [tuple(x) for x in config['ionic_channels']]
    unique = list(dict.fromkeys((n, l, abs(m)) for n, l, m in labels))
    columns = [unique.index((n, l, abs(m))) for n, l, m in labels]
    ion = Ionic(base, {m for n, l, m in unique})
    contractor = SurfaceContractor(base, ion, labels, unique, columns, True, h.transform, DEVICE)
    pulse = Pulse(**config['pulses'][0]['pulse'])
    avec = lambda t: np.array([0., 0., float(pulse.vector(t))])
    return h, base, ion, contractor, avec


def test_contraction_matches_reference():
    g = golden('volkov')
    h, base, ion, contractor, avec = _setup()
    assert ion.na == int(g['nion']) and contractor.outerstates == [tuple(x) for x in g['outerstates']]
    for i in range(len(g['times'])):
        q = contractor(g['chi'][i], g['frames'][i])
        np.testing.assert_allclose(q, g['q'][i], rtol=1e-12, atol=1e-13)


def test_volkov_accumulation_matches_reference():
    from laqphysics_b200.streaming_surface import VolkovAccumulator
    g = golden('volkov')
    h, base, ion, contractor, avec = _setup()
    np.testing.assert_allclose(np.array([avec(t) for t in g['times']]), g['avec'], atol=1e-15)
    acc = VolkovAccumulator(contractor, CONFIG, avec, device=DEVICE)
    np.testing.assert_allclose(acc.tests, g['tests'], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(acc.harmonics, g['harmonics'], rtol=1e-13, atol=1e-15)
    for i, t in enumerate(g['times']):
        acc.add(i, t, g['q'][i])
    np.testing.assert_allclose(acc.amplitude.cpu().numpy(), g['amplitude'], rtol=3e-12, atol=3e-12)


def test_accumulator_checkpoint_restore_continues_identically():
    from laqphysics_b200.streaming_surface import VolkovAccumulator
    g = golden('volkov')
    h, base, ion, contractor, avec = _setup()
    acc = VolkovAccumulator(contractor, CONFIG, avec, device=DEVICE)
    for i in range(8):
        acc.add(i, g['times'][i], g['q'][i])
    saved = {k: np.array(v, copy=True) for k, v in acc.payload().items()}
    resumed = VolkovAccumulator(contractor, CONFIG, avec, device=DEVICE)
    resumed.restore(saved)
    for i in range(8, len(g['times'])):
        resumed.add(i, g['times'][i], g['q'][i])
    np.testing.assert_allclose(resumed.amplitude.cpu().numpy(), g['amplitude'], rtol=3e-12, atol=3e-12)
    with pytest.raises(ValueError, match='nonsequential'):
        resumed.add(3, 0., g['q'][0])


def test_fused_surface_sample_from_device_state():
    """flux frame of a device state -> contraction -> accumulation, no host copies,
    equals the host flux + reference-order contraction."""
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.streaming_surface import SurfaceSampler, VolkovAccumulator
    from laqphysics_b200.workloads import seeded_state
    g = golden('volkov')
    h, base, ion, contractor, avec = _setup()
    op = B200Hamiltonian(h, DEVICE)
    sampler = SurfaceSampler(op, contractor, VolkovAccumulator(contractor, CONFIG, avec, device=DEVICE))
    ref_acc = VolkovAccumulator(contractor, CONFIG, avec, device=DEVICE)
    for i, t in enumerate(g['times'][:5]):
        x = seeded_state(h.size, 100 + i)
        q = sampler.record(i, t, op.state(x), avec(t), g['chi'][i])
        q_ref = contractor(g['chi'][i], h.flux(x, avec(t)))
        np.testing.assert_allclose(q.cpu().numpy(), q_ref, rtol=1e-11, atol=1e-13)
        ref_acc.add(i, t, q_ref)
    np.testing.assert_allclose(sampler.accumulator.amplitude.cpu().numpy(), ref_acc.amplitude.cpu().numpy(),
                               rtol=1e-11, atol=1e-13)


def test_sampler_keeps_projected_and_raw_history_in_shards(tmp_path):
    """SurfaceSampler with the reference's 'projected' and 'raw_shards' storage: every q and
    every flux frame lands in capped NPY shards (surface_storage.ShardedArray) that read back
    equal to the device values and to the host flux."""
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.streaming_surface import SurfaceSampler, VolkovAccumulator
    from laqphysics_b200.surface_storage import ShardedArray, load_flux
    from laqphysics_b200.workloads import seeded_state
    g = golden('volkov')
    h, base, ion, contractor, avec = _setup()
    op = B200Hamiltonian(h, DEVICE)
    count = 5
    frame_shape = tuple(op.surface.frame(op.state(seeded_state(h.size, 1)), avec(0.)).shape)
    q_shape = tuple(contractor.contract(torch.as_tensor(g['chi'][0], device=DEVICE),
                                        op.surface.frame(op.state(seeded_state(h.size, 1)), avec(0.))).shape)
    raw = ShardedArray(tmp_path / 'run' / 'flux_shards', (count, *frame_shape), mode='w+', max_file_bytes=2 * 16 * int(np.prod(frame_shape)) + 4200)
    projected = ShardedArray(tmp_path / 'run' / 'projected', (count, *q_shape), mode='w+', max_file_bytes=100000)
    sampler = SurfaceSampler(op, contractor, VolkovAccumulator(contractor, CONFIG, avec, device=DEVICE),
                             projected=projected, raw=raw)
    qs = []
    for i, t in enumerate(g['times'][:count]):
        x = seeded_state(h.size, 100 + i)
        qs.append(sampler.record(i, t, op.state(x), avec(t), g['chi'][i]).cpu().numpy())
    raw.close()
    projected.close()
    flux = load_flux(tmp_path / 'run')
    assert len(list((tmp_path / 'run' / 'flux_shards').glob('part_*.npy'))) == 3
    for i, t in enumerate(g['times'][:count]):
        np.testing.assert_allclose(flux[i], h.flux(seeded_state(h.size, 100 + i), avec(t)), rtol=1e-12, atol=1e-14)
    np.testing.assert_array_equal(ShardedArray(tmp_path / 'run' / 'projected')[:], np.array(qs))


def test_one_launch_sample_equals_the_three_launch_chain():
    """he_sample_record (flux frame, contraction and Volkov update in one cooperative launch
    whose CTAs wait for each other's partial sums) against he_flux -> he_surface_contract ->
    he_volkov_add on the same device states and channel functions: frames bit for bit, q
    and amplitudes to rounding (q sums per CTA in a different order), on a grid of several
    CTAs; the bounded wait reports no time-out."""
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.streaming_surface import SurfaceSampler, VolkovAccumulator
    from laqphysics_b200.workloads import seeded_state
    config = dict(CONFIG, radial={'edges': list(range(0, 21, 2)), 'order': 6, 'tail': 8, 'ecs_angle': .3},
                  lmax=2, total_Lmax=2, cutoff_radii=[10, 14], surface=16., spectrum_energy=[.2, 3., 240],
                  spectrum={'theta_points': 16, 'phi_points': 1})
    h, base, ion, contractor, avec = _setup(config)
    op = B200Hamiltonian(h, DEVICE)
    raw1, raw3 = {}, {}
    one = SurfaceSampler(op, contractor, VolkovAccumulator(contractor, config, avec, device=DEVICE), raw=raw1)
    three = SurfaceSampler(op, contractor, VolkovAccumulator(contractor, config, avec, device=DEVICE), raw=raw3,
                           fused=False)
    assert one.fused.grid > 1 and three.fused is None
    rng = np.random.default_rng(3)
    chi = torch.as_tensor(rng.normal(size=(ion.na * h.n, len(contractor.unique))) +
                          1j * rng.normal(size=(ion.na * h.n, len(contractor.unique))), device=DEVICE)
    for i in range(6):
        t = .25 * i
        state = op.state(seeded_state(h.size, 40 + i))
        q1 = one.record(i, t, state, avec(t), chi)
        q3 = three.record(i, t, state, avec(t), chi)
        assert torch.equal(raw1[i], raw3[i])
        scale = float(torch.max(torch.abs(q3)))
        assert float(torch.max(torch.abs(q1 - q3))) <= 1e-14 * scale
    a1, a3 = one.accumulator.amplitude, three.accumulator.amplitude
    assert float(torch.max(torch.abs(a1 - a3))) <= 1e-13 * float(torch.max(torch.abs(a3)))
    one.fused.status()


def test_sample_wait_that_runs_out_reports_and_leaves_the_device_usable():
    """The one-launch sample's only inter-CTA wait is bounded: with the test hook making the
    CTAs wait for an arrival that never comes, the record returns, he_sample_status reports
    HE_ERR_DEVICE once, and the next records on the same device give the three-launch
    chain's q again."""
    from laqphysics_b200._lib import LIB
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.streaming_surface import SurfaceSampler, VolkovAccumulator
    from laqphysics_b200.workloads import seeded_state
    g = golden('volkov')
    h, base, ion, contractor, avec = _setup()
    op = B200Hamiltonian(h, DEVICE)
    state = op.state(seeded_state(h.size, 7))
    stalled = SurfaceSampler(op, contractor, VolkovAccumulator(contractor, CONFIG, avec, device=DEVICE))
    assert LIB.he_sample_set_wait_extra(stalled.fused.handle, 1) == 0
    stalled.record(0, 0., state, avec(0.), g['chi'][0])
    torch.cuda.synchronize()
    with pytest.raises(RuntimeError, match='ran out'):
        stalled.fused.status()
    stalled.fused.status()                       # reported once
    one = SurfaceSampler(op, contractor, VolkovAccumulator(contractor, CONFIG, avec, device=DEVICE))
    three = SurfaceSampler(op, contractor, VolkovAccumulator(contractor, CONFIG, avec, device=DEVICE), fused=False)
    for i, t in enumerate(g['times'][:3]):
        q1 = one.record(i, t, state, avec(t), g['chi'][i])
        q3 = three.record(i, t, state, avec(t), g['chi'][i])
        assert float(torch.max(torch.abs(q1 - q3))) <= 1e-14 * float(torch.max(torch.abs(q3)))
    one.fused.status()
