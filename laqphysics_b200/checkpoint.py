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


def capped_npz(path, max_file_bytes=DEFAULT_FILE_BYTES, **arrays):
    """np.savez to a temporary file beside `path`, refused above `max_file_bytes` (checked
    before and after writing), then renamed over `path`."""
    path = Path(path)
    limit = int(max_file_bytes)
    if limit <= 0:
        raise ValueError('file cap must be positive')
    estimate = sum(np.asarray(v).nbytes + 1024 for v in arrays.values()) + 4096
    if estimate > limit:
        raise ValueError(f'{path.name}: checkpoint needs about {estimate} bytes, above file cap {limit}')
    temporary = path.with_name(path.stem + '.tmp.npz')
    np.savez(temporary, **arrays)
    if temporary.stat().st_size > limit:
        temporary.unlink()
        raise ValueError('NPZ exceeds configured file cap')
    os.replace(temporary, path)


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
