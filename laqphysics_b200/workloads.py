"""Named synthetic workloads (grids, channel sets, pulses) used by bench.py and tests.

Each reproduces a reference-style setup (python/run3d.py:23-39: ``make_grid`` +
``Helium`` + ``CoupledHelium``) at a stated size.  Mapping choices the reference's
grid cannot express literally are spelled out in the docstrings.
"""
import numpy as np

from .coupled_angular import CoupledHelium
from .fedvr import make_grid
from .helium3d import Helium
from .pulses import Pulse


def coupled(edges, order, lmax, total_Lmax, ecs_angle=0., tail=0, alpha=1., cutoff_radii=None):
    grid = make_grid(edges, order, ecs_angle=ecs_angle, tail=tail, alpha=alpha)
    return CoupledHelium(Helium(grid, lmax, M=0, cutoff_radii=cutoff_radii), total_Lmax)


def hpsi_microbench(tail=20, ecs_angle=.35):
    """H·psi microbenchmark grid: 60 finite elements of order 9 (10 Lobatto nodes each,
    541 points) on [0, 120] a.u., then an infinite exterior-scaled Laguerre tail of
    ``tail`` points from 120 a.u. at theta = 0.35 (alpha = 1; the reference's irECS
    has no finite outer edge, so "box 150" maps to this tail).  Coupled channels
    l1, l2 <= 5, L <= 3, M = 0 -> nc = 43; origin removed -> n = 560 at tail = 20,
    N = n^2 nc = 13 484 800 amplitudes.  Coulomb cut between 80 and 95 a.u."""
    return coupled(np.linspace(0, 120, 61), 9, 5, 3, ecs_angle=ecs_angle, tail=tail, cutoff_radii=(80., 95.))


def arnoldi_small(tail=12):
    """Plain FP64 Arnoldi grid: 15 elements of order 8 on [0, 25] a.u. + ECS tail of
    ``tail`` points from 25 a.u. (theta 0.3, alpha 1) -> n = 132 at tail 12; coupled
    l1, l2 <= 3, L <= 2, M = 0 -> nc = 17; N = 296 208.  Coulomb cut 18..22 a.u."""
    return coupled(np.linspace(0, 25, 16), 8, 3, 2, ecs_angle=.3, tail=tail, cutoff_radii=(18., 22.))


def arnoldi_small_real(tail=12):
    """Real (unscaled, theta = 0) twin of :func:`arnoldi_small`, same nodes count, for the
    ground-state solve (python/run3d.py:24-25 builds both grids from one config)."""
    return coupled(np.linspace(0, 25, 16), 8, 3, 2, ecs_angle=0., tail=tail, cutoff_radii=(18., 22.))


def adjoint_grid(tail=12, ecs_angle=.3):
    """Adjoint-gradient grid: the Arnoldi grid widened to l1, l2 <= 4 (L <= 2, M = 0)."""
    return coupled(np.linspace(0, 25, 16), 8, 4, 2, ecs_angle=ecs_angle, tail=tail, cutoff_radii=(18., 22.))


def length_pulse():
    """Linear sin^2 pulse, omega 1.6 a.u., 10 cycles, peak field 0.01 a.u."""
    return Pulse(omega=1.6, cycles=10, field=.01)


def seeded_state(size, seed, dtype=np.complex128):
    """Seed-drawn complex Gaussian, normalised."""
    rng = np.random.default_rng(seed)
    x = rng.normal(size=size) + 1j * rng.normal(size=size)
    return (x / np.linalg.norm(x)).astype(dtype)


def hpsi_flop_parts(h):
    """Algorithmic real flops of one complex H·psi (complex MAC = 8 flops), by part:
    kinetic on both electrons, Coulomb edges (complex coefficient x complex radial x
    complex psi = 2 complex products), length-gauge dipole edges and the diagonal."""
    n2 = h.n * h.n
    nnz = int(h.ptr[-1])
    return {'kinetic': 2 * nnz * h.n * h.nc * 8, 'coulomb': len(h.vc) * n2 * 14, 'dipole': len(h.dc) * n2 * 14,
            'diagonal': h.nc * n2 * 8}


def hpsi_flops(h):
    """Total algorithmic real flops of one complex H·psi (see hpsi_flop_parts)."""
    return sum(hpsi_flop_parts(h).values())
