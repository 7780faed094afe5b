"""Sharded surface storage (laqphysics_b200.surface_storage) against shards written by the
reference's own ShardedArray (tests/golden/shards, made by tests/golden/make_golden.py):
same manifest, same shard files byte for byte, and the reference's own boundary/reopen
case (tests/test_streaming_surface.py:22-28)."""
from pathlib import Path

import numpy as np
import pytest

from laqphysics_b200.surface_storage import ShardedArray, load_flux

GOLDEN = Path(__file__).resolve().parent / 'golden'


def test_reads_reference_shards():
    values = np.load(GOLDEN / 'shards_values.npz')['values']
    a = ShardedArray(GOLDEN / 'shards')
    assert a.shape == values.shape and a.frames_per_file == 3
    np.testing.assert_array_equal(a[:], values)
    np.testing.assert_array_equal(a[[6, 0, 4]], values[[6, 0, 4]])
    np.testing.assert_array_equal(a[-1], values[-1])
    with pytest.raises(ValueError):
        a[0] = values[0]


def test_writes_the_reference_layout_byte_for_byte(tmp_path):
    values = np.load(GOLDEN / 'shards_values.npz')['values']
    a = ShardedArray(tmp_path / 'shards', values.shape, mode='w+', max_file_bytes=4400)
    for i in reversed(range(len(a))):
        a[i] = values[i]
    a.close()
    ours = sorted(p.name for p in (tmp_path / 'shards').iterdir())
    assert ours == sorted(p.name for p in (GOLDEN / 'shards').iterdir())
    for name in ours:
        assert (tmp_path / 'shards' / name).read_bytes() == (GOLDEN / 'shards' / name).read_bytes(), name


def test_shards_cross_boundaries_reopen_and_respect_the_cap(tmp_path):
    shape = (23, 17, 7)
    expected = np.arange(np.prod(shape)).reshape(shape) * (1 + 2j)
    a = ShardedArray(tmp_path / 'a', shape, mode='w+', max_file_bytes=12000)
    for i in reversed(range(len(a))):
        a[i] = expected[i]
    a.close()
    b = ShardedArray(tmp_path / 'a')
    np.testing.assert_array_equal(b[:], expected)
    parts = list((tmp_path / 'a').glob('part*.npy'))
    assert len(parts) > 1 and all(p.stat().st_size <= 12000 for p in parts)
    c = ShardedArray(tmp_path / 'a', mode='r+')
    c[5] = -expected[5]
    c.close()
    np.testing.assert_array_equal(ShardedArray(tmp_path / 'a')[5], -expected[5])
    with pytest.raises(FileExistsError):
        ShardedArray(tmp_path / 'a', shape, mode='w+', max_file_bytes=12000)
    with pytest.raises(ValueError):
        ShardedArray(tmp_path / 'big', (2, 1000), mode='w+', max_file_bytes=5000)
    with pytest.raises(ValueError):
        ShardedArray(tmp_path / 'tiny', (2, 1), mode='w+', max_file_bytes=4096)


def test_load_flux_finds_sharded_history(tmp_path):
    out = tmp_path / 'run'
    a = ShardedArray(out / 'flux_shards', (4, 2, 3, 1), mode='w+', max_file_bytes=8192)
    a[0] = np.ones((2, 3, 1))
    a.close()
    flux = load_flux(out)
    assert len(flux) == 4 and np.all(flux[0] == 1)
    with pytest.raises(FileNotFoundError):
        load_flux(tmp_path / 'empty')
