"""Run checkpoints in the reference's format (python/run3d.py:164-172, written through the
atomic size-capped NPZ of python/surface_storage.py:18-26): keys, dtypes, round trip, cap."""
import numpy as np
import pytest

from laqphysics_b200.checkpoint import CHECKPOINT_KEYS, read_checkpoint, write_checkpoint

# the keys run3d.save() writes, in its order
REFERENCE_KEYS = ['psi', 'step', 'signature', 'ground_energy', 'ground', 'ground_residual', 'surface_generation',
                  'maximum_linear_residual_all_segments', 'linear_iterations_all_segments']


def test_checkpoint_keys_round_trip_and_cap(tmp_path):
    assert list(CHECKPOINT_KEYS) == REFERENCE_KEYS
    rng = np.random.default_rng(1)
    psi = rng.normal(size=300) + 1j * rng.normal(size=300)
    ground = rng.normal(size=300) + 0j
    path = tmp_path / 'checkpoint.npz'
    write_checkpoint(path, psi, 17, 'abc', -2.9, ground, 1e-11, 3, 2e-12, 456)
    with np.load(path) as data:
        assert list(data.files) == REFERENCE_KEYS
        assert data['psi'].dtype == np.complex128 and data['step'].dtype.kind == 'i'
    back = read_checkpoint(path)
    np.testing.assert_array_equal(back['psi'], psi)
    assert int(back['step']) == 17 and str(back['signature']) == 'abc' and int(back['surface_generation']) == 3
    assert not (tmp_path / 'checkpoint.tmp.npz').exists()
    with pytest.raises(ValueError):
        write_checkpoint(tmp_path / 'big.npz', psi, 1, 's', 0., ground, 0., max_file_bytes=1000)
    assert not (tmp_path / 'big.npz').exists()
