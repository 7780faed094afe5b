"""Per-sample surface data in size-capped NPY shards (the reference's on-disk layout).

The reference's ``raw_shards`` and ``projected`` storage modes (python/run3d.py:84-141,
python/streaming_surface.py:187-190, 255, 267) keep one frame per surface sample in a folder
of NPY files, each at most a byte cap (python/surface_storage.py:28-74).  The folder holds

* ``array.json``: {"shape", "dtype" (numpy dtype string), "frames_per_file",
  "max_file_bytes"}, JSON with indent 2 and a trailing newline, written atomically;
* ``part_000000.npy``, ``part_000001.npy``, ...: frames_per_file consecutive frames each
  (the last shard holds the remainder), where frames_per_file = (cap - 4096) // frame bytes
  leaves 4096 bytes for the NPY header.

Those files are an interface: the reference's tools (``load_flux``, the projected-mode
quadrature) and this engine read each other's runs, and the tests check the files byte for
byte.  The code is organised as a pure layout (which shard and row hold a frame, how many
rows a shard has) and an accessor that keeps one shard memory-mapped at a time.  Frames may
be device tensors; they are copied to the host when stored.
"""
import json
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

DEFAULT_FILE_BYTES = 4_000_000_000
HARD_FILE_BYTES = 5_000_000_000
HEADER_RESERVE = 4096
MANIFEST = 'array.json'


def atomic_json(path, value):
    """Write `value` as indented JSON beside `path`, then rename it into place."""
    path = Path(path)
    staged = path.parent / (path.name + '.tmp')
    staged.write_text(json.dumps(value, indent=2) + '\n')
    os.replace(staged, path)


def file_limit(value=DEFAULT_FILE_BYTES):
    """A per-file byte cap: above the header reserve and at most 5 GB (decimal)."""
    cap = int(value)
    if cap <= HEADER_RESERVE or cap > HARD_FILE_BYTES:
        raise ValueError(f'a file cap of {cap} bytes is outside ({HEADER_RESERVE}, {HARD_FILE_BYTES}]')
    return cap


@dataclass(frozen=True)
class ShardLayout:
    """Where frame k of a (frames, ...) array lives: shard k // per_file, row k % per_file."""
    shape: tuple
    dtype: np.dtype
    per_file: int
    cap: int

    @classmethod
    def plan(cls, shape, dtype, cap):
        shape, dtype, cap = tuple(int(s) for s in shape), np.dtype(dtype), file_limit(cap)
        frame_bytes = dtype.itemsize * int(np.prod(shape[1:], dtype=np.int64))
        per_file = (cap - HEADER_RESERVE) // frame_bytes
        if per_file < 1:
            raise ValueError(f'a single frame ({frame_bytes} bytes) does not fit the {cap}-byte file cap')
        return cls(shape, dtype, per_file, cap)

    @classmethod
    def read(cls, folder):
        meta = json.loads((Path(folder) / MANIFEST).read_text())
        return cls(tuple(meta['shape']), np.dtype(meta['dtype']), int(meta['frames_per_file']),
                   int(meta['max_file_bytes']))

    def manifest(self):
        return {'shape': list(self.shape), 'dtype': self.dtype.str, 'frames_per_file': self.per_file,
                'max_file_bytes': self.cap}

    @property
    def frames(self):
        return self.shape[0]

    def locate(self, frame):
        """(shard, row) of a frame index; negative indices count from the end."""
        k = frame + self.frames if frame < 0 else frame
        if not 0 <= k < self.frames:
            raise IndexError(f'frame {frame} outside 0..{self.frames - 1}')
        return divmod(k, self.per_file)

    def rows(self, shard):
        return min(self.per_file, self.frames - shard * self.per_file)

    @staticmethod
    def filename(shard):
        return f'part_{shard:06d}.npy'


class ShardedArray:
    """A (frames, ...) array in capped NPY shards.  mode 'w+' creates the folder (and
    refuses an existing one), 'r+' reopens it for writing, 'r' reads.  Index by int,
    slice or a list of ints."""

    def __init__(self, folder, shape=None, dtype=np.complex128, mode='r', max_file_bytes=DEFAULT_FILE_BYTES):
        if mode not in ('r', 'r+', 'w+'):
            raise ValueError(f'unknown mode {mode!r}')
        self.folder, self.mode = Path(folder), mode
        if mode == 'w+':
            if (self.folder / MANIFEST).exists():
                raise FileExistsError(self.folder / MANIFEST)
            self.layout = ShardLayout.plan(shape, dtype, max_file_bytes)
            self.folder.mkdir(parents=True, exist_ok=True)
            atomic_json(self.folder / MANIFEST, self.layout.manifest())
        else:
            self.layout = ShardLayout.read(self.folder)
        self._open = (None, None)         # (shard number, memory map)

    # the reference's attribute names
    shape = property(lambda self: self.layout.shape)
    dtype = property(lambda self: self.layout.dtype)
    frames_per_file = property(lambda self: self.layout.per_file)
    limit = property(lambda self: self.layout.cap)

    def __len__(self):
        return self.layout.frames

    def _shard(self, shard):
        """The memory map of one shard (created full-size on first write)."""
        current, array = self._open
        if current == shard:
            return array
        self.flush()
        path = self.folder / ShardLayout.filename(shard)
        if path.exists():
            array = np.load(path, mmap_mode='r' if self.mode == 'r' else 'r+')
        elif self.mode == 'r':
            raise FileNotFoundError(path)
        else:
            array = np.lib.format.open_memmap(path, mode='w+', dtype=self.layout.dtype,
                                              shape=(self.layout.rows(shard), *self.layout.shape[1:]))
            if path.stat().st_size > self.layout.cap:
                raise RuntimeError(f'{path.name} is {path.stat().st_size} bytes, above the {self.layout.cap}-byte cap')
        self._open = (shard, array)
        return array

    def _frame(self, k):
        shard, row = self.layout.locate(int(k))
        return self._shard(shard)[row]

    def __getitem__(self, index):
        if isinstance(index, slice):
            return np.array([self._frame(k) for k in range(*index.indices(len(self)))])
        if np.isscalar(index):
            return self._frame(index)
        return np.array([self._frame(k) for k in index])

    def __setitem__(self, index, value):
        if self.mode == 'r':
            raise ValueError(f'{self.folder} is open read-only')
        if hasattr(value, 'detach'):      # a device frame
            value = value.detach().cpu().numpy()
        shard, row = self.layout.locate(int(index))
        self._shard(shard)[row] = value

    def flush(self):
        _, array = self._open
        if array is not None and self.mode != 'r':
            array.flush()

    def close(self):
        self.flush()
        self._open = (None, None)


def load_flux(out):
    """The raw surface history of a run folder: a monolithic flux.npy or flux_shards/."""
    out = Path(out)
    if (out / 'flux.npy').exists():
        return np.load(out / 'flux.npy', mmap_mode='r')
    if (out / 'flux_shards' / MANIFEST).exists():
        return ShardedArray(out / 'flux_shards')
    raise FileNotFoundError(f'{out} holds no raw surface history (neither flux.npy nor flux_shards/); '
                            'online-spectrum runs do not keep one')
