import os
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / 'tests' / 'golden'
sys.path.insert(0, str(REPO))
os.environ.setdefault('OMP_NUM_THREADS', str(min(8, os.cpu_count() or 1)))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (B200) and runs the sm_100a kernels')


def golden(name):
    with np.load(GOLDEN / f'{name}.npz', allow_pickle=False) as data:
        return {k: data[k] for k in data.files}


class Tables:
    """Table object rebuilt from a golden fixture (the reference's own arrays)."""

    def __init__(self, g):
        for key, value in g.items():
            if key.startswith('t_'):
                setattr(self, key[2:], value)
        self.shape = tuple(int(s) for s in g['shape'])
        self.n, _, self.nc = self.shape
        self.size = int(np.prod(self.shape))
        self.diag = np.asfortranarray(self.diag)
        self.rad = np.asfortranarray(self.rad)
        self.dcoef = np.asfortranarray(self.dcoef)


@pytest.fixture(scope='session')
def gold():
    return golden


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
