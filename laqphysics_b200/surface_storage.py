"""Size-capped NPY shards for per-sample surface data, in the reference's on-disk format.

The reference's ``raw_shards`` and ``projected`` storage modes (python/run3d.py:84-141,
python/streaming_surface.py:187-190, 255, 267) keep one frame per surface sample in a folder
of NPY files no larger than a byte cap (python/surface_storage.py:28-74): a manifest
``array.json`` (shape, dtype string, frames per file, byte cap, written atomically) and
shards ``part_000000.npy``, ``part_000001.npy``, ... each holding ``frames_per_file``
consecutive frames (the last one the remainder), frames_per_file = (cap - 4096) // frame
bytes.  This module writes and reads exactly that layout, so the reference's tools
(``load_flux``, projected-mode quadrature) read runs of this engine and the other way
round.  Frames may be device tensors: they are copied to the host when stored.
"""
import json
import os
from pathlib import Path

import numpy as np

DEFAULT_FILE_BYTES = 4_000_000_000
HARD_FILE_BYTES = 5_000_000_000


def atomic_json(path, value):
    """JSON (indent 2, trailing newline) through a temporary file renamed over `path`."""
    path = Path(path)
    temporary = path.with_name(path.name + '.tmp')
    temporary.write_text(json.dumps(value, indent=2) + '\n')
    os.replace(temporary, path)


def file_limit(value=DEFAULT_FILE_BYTES):
    value = int(value)
    if not 4096 < value <= HARD_FILE_BYTES:
        raise ValueError('max_file_bytes must be >4096 and <=5,000,000,000 (decimal bytes)')
    return value


class ShardedArray:
    """A (frames, ...) array stored as capped NPY shards; mode 'w+' creates the folder,
    'r+' reopens it for writing, 'r' reads.  Indexing by int, slice or index list."""

    def __init__(self, folder, shape=None, dtype=np.complex128, mode='r', max_file_bytes=DEFAULT_FILE_BYTES):
        self.folder, self.mode = Path(folder), mode
        self._part, self._array = None, None
        manifest = self.folder / 'array.json'
        if mode == 'w+':
            if manifest.exists():
                raise FileExistsError(manifest)
            self.folder.mkdir(parents=True, exist_ok=True)
            self.shape, self.dtype = tuple(int(s) for s in shape), np.dtype(dtype)
            self.limit = file_limit(max_file_bytes)
            frame = int(np.prod(self.shape[1:])) * self.dtype.itemsize
            self.frames_per_file = (self.limit - 4096) // frame
            if self.frames_per_file < 1:
                raise ValueError('one array frame exceeds file cap; refine storage layout')
            atomic_json(manifest, {'shape': self.shape, 'dtype': self.dtype.str,
                                   'frames_per_file': self.frames_per_file, 'max_file_bytes': self.limit})
        else:
            meta = json.loads(manifest.read_text())
            self.shape, self.dtype = tuple(meta['shape']), np.dtype(meta['dtype'])
            self.frames_per_file, self.limit = int(meta['frames_per_file']), int(meta['max_file_bytes'])

    def __len__(self):
        return self.shape[0]

    def _row(self, index):
        """Open the shard holding frame `index`; its row there."""
        if index < 0:
            index += len(self)
        if not 0 <= index < len(self):
            raise IndexError(index)
        part = index // self.frames_per_file
        if part != self._part:
            self.flush()
            self._array = None
            path = self.folder / f'part_{part:06d}.npy'
            if path.exists():
                self._array = np.load(path, mmap_mode='r' if self.mode == 'r' else 'r+')
            elif self.mode == 'r':
                raise FileNotFoundError(path)
            else:
                rows = min(self.frames_per_file, len(self) - part * self.frames_per_file)
                self._array = np.lib.format.open_memmap(path, mode='w+', dtype=self.dtype,
                                                        shape=(rows, *self.shape[1:]))
                if path.stat().st_size > self.limit:
                    raise RuntimeError('shard exceeded file cap')
            self._part = part
        return index % self.frames_per_file

    def __getitem__(self, index):
        if isinstance(index, slice):
            return np.array([self[i] for i in range(*index.indices(len(self)))])
        if not np.isscalar(index):
            return np.array([self[int(i)] for i in index])
        row = self._row(int(index))      # opens the shard first
        return self._array[row]

    def __setitem__(self, index, value):
        if self.mode == 'r':
            raise ValueError('read-only array')
        if hasattr(value, 'detach'):   # a device frame
            value = value.detach().cpu().numpy()
        row = self._row(int(index))
        self._array[row] = value

    def flush(self):
        if self._array is not None and self.mode != 'r':
            self._array.flush()

    def close(self):
        self.flush()
        self._array, self._part = None, None


def load_flux(out):
    """The raw surface history of a run folder: monolithic flux.npy or flux_shards."""
    out = Path(out)
    if (out / 'flux.npy').exists():
        return np.load(out / 'flux.npy', mmap_mode='r')
    if (out / 'flux_shards' / 'array.json').exists():
        return ShardedArray(out / 'flux_shards')
    raise FileNotFoundError('No raw surface history; an online spectrum run intentionally does not write flux.npy')
