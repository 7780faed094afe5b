"""Run checkpoints and spectra in the reference's on-disk formats.

The reference's driver stores its restart point as one NPZ with the keys of
python/run3d.py:164-172 (psi, step, signature, ground_energy, ground, ground_residual,
surface_generation, maximum_linear_residual_all_segments, linear_iterations_all_segments)
and the tSURFF spectrum with the keys of python/streaming_surface.py:74-82, both through an
atomic, size-capped write (python/surface_storage.py:18-26).  Writing the same keys, dtypes
and layout (psi in Fortran order, complex128) lets the reference's tools (restart,
extract_run, spectrum_report) read runs of this engine unchanged.
"""
import os
from pathlib import Path

import numpy as np
import torch

DEFAULT_FILE_BYTES = 4_000_000_000
CHECKPOINT_KEYS = ('psi', 'step', 'signature', 'ground_energy', 'ground', 'ground_residual', 'surface_generation',
                   'maximum_linear_residual_all_segments', 'linear_iterations_all_segments')


def _npz_estimate(arrays):
    """Upper estimate of an uncompressed NPZ: the payloads plus 1 KiB per member for its
    NPY header and zip entry, plus 4 KiB for the zip directory."""
    return 4096 + sum(1024 + np.asarray(v).nbytes for v in arrays.values())


def capped_npz(path, max_file_bytes=DEFAULT_FILE_BYTES, **arrays):
    """Write an uncompressed NPZ atomically, refusing it above `max_file_bytes`: the size
    is estimated before writing and measured after, then the staged file is renamed over
    `path` (a refused write leaves `path` untouched)."""
    path = Path(path)
    cap = int(max_file_bytes)
    if cap <= 0:
        raise ValueError(f'file cap must be positive, got {cap}')
    needed = _npz_estimate(arrays)
    if needed > cap:
        raise ValueError(f'{path.name}: about {needed} bytes would exceed the {cap}-byte file cap')
    staged = path.parent / (path.stem + '.tmp.npz')
    np.savez(staged, **arrays)
    written = staged.stat().st_size
    if written > cap:
        staged.unlink()
        raise ValueError(f'{path.name}: {written} bytes written, above the {cap}-byte file cap')
    os.replace(staged, path)


def write_checkpoint(path, psi, step, signature, ground_energy, ground, ground_residual, surface_generation=-1,
                     maximum_linear_residual=0., linear_iterations=0, max_file_bytes=DEFAULT_FILE_BYTES):
    """Restart point of a run; psi (and ground) may be device tensors or host arrays."""
    host = lambda x: x.detach().cpu().numpy() if torch.is_tensor(x) else np.asarray(x)
    capped_npz(path, max_file_bytes, psi=host(psi).astype(np.complex128), step=int(step), signature=signature,
               ground_energy=ground_energy, ground=host(ground), ground_residual=ground_residual,
               surface_generation=int(surface_generation), maximum_linear_residual_all_segments=maximum_linear_residual,
               linear_iterations_all_segments=int(linear_iterations))


def read_checkpoint(path, device=None):
    """The checkpoint's fields as a dict; with `device`, psi comes back as a device tensor."""
    with np.load(path, allow_pickle=False) as data:
        out = {k: data[k] for k in data.files}
    missing = [k for k in CHECKPOINT_KEYS if k not in out]
    if missing:
        raise ValueError(f'not a run checkpoint (missing {missing})')
    if device is not None:
        out['psi'] = torch.as_tensor(out['psi'], dtype=torch.complex128, device=device)
    return out
