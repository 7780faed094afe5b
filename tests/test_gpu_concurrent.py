"""Instances of different operators stepped concurrently (laqphysics_b200.concurrent) give
bit-identical results to stepping each alone."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEVICE = 'cuda:0'


def test_concurrent_uneven_instances_match_single_steps():
    from laqphysics_b200.concurrent import ConcurrentStepper
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.torch_backend import FieldSchedule, step
    from laqphysics_b200.workloads import coupled, seeded_state
    grids = [(np.linspace(0, 12, 7), 5, 1, 1, 8), (np.linspace(0, 16, 9), 6, 2, 2, 10), (np.linspace(0, 10, 6), 4, 2, 1, 6)]
    engines, schedules, states = [], [], []
    for k, (edges, order, lmax, L, tail) in enumerate(grids):
        h = coupled(edges, order, lmax, L, ecs_angle=.3, tail=tail, cutoff_radii=(4., 5.))
        e = B200Hamiltonian(h, DEVICE)
        amp = .02 * (k + 1)
        schedules.append(FieldSchedule(e, lambda t, a=amp: (0., 0., a * np.sin(t)), velocity=False))
        x = seeded_state(h.size, 70 + k)
        states.append(e.state(x / np.linalg.norm(x)))
        engines.append(e)
    stepper = ConcurrentStepper(schedules, DEVICE)
    together = states
    alone = [s.clone() for s in states]
    for i in range(3):
        together, infos = stepper.step(together, i * .01, .01, 1e-10, 20)
        alone = [step(sch, x, i * .01, .01, 1e-10, 20)[0] for sch, x in zip(schedules, alone)]
    torch.cuda.synchronize()
    for a, b in zip(together, alone):
        np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())
    stepper.close()


def test_concurrent_cf4_steps_match_single_steps():
    """CF4 + Pade/GMRES steps of instances of different operators, each with its own
    separable preconditioner, concurrently and one by one: identical."""
    from laqphysics_b200.concurrent import ConcurrentStepper
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.implicit import SeparablePreconditioner, cf4_step
    from laqphysics_b200.torch_backend import FieldSchedule
    from laqphysics_b200.workloads import coupled, seeded_state
    grids = [(np.linspace(0, 12, 7), 5, 1, 1, 8), (np.linspace(0, 16, 9), 6, 2, 2, 10)]
    schedules, states, avecs = [], [], []
    for k, (edges, order, lmax, L, tail) in enumerate(grids):
        h = coupled(edges, order, lmax, L, ecs_angle=.3, tail=tail, cutoff_radii=(4., 5.))
        e = B200Hamiltonian(h, DEVICE)
        e.separable = SeparablePreconditioner(e, 'complex128' if k == 0 else 'complex64')
        avecs.append(lambda t, a=.1 * (k + 1): np.array([0., 0., a * np.sin(t)]))
        schedules.append(FieldSchedule(e, avecs[-1], velocity=True))
        x = seeded_state(h.size, 80 + k)
        states.append(e.state(x / np.linalg.norm(x)))
    stepper = ConcurrentStepper(schedules, DEVICE)
    together = states
    alone = [s.clone() for s in states]
    for i in range(2):
        together, _ = stepper.cf4(together, avecs, i * .02, .02, [-2.9, -2.8], 1e-11)
        alone = [cf4_step(sch.engine, x, av, i * .02, .02, er, 1e-11)[0]
                 for sch, x, av, er in zip(schedules, alone, avecs, [-2.9, -2.8])]
    torch.cuda.synchronize()
    for a, b in zip(together, alone):
        np.testing.assert_array_equal(a.cpu().numpy(), b.cpu().numpy())
    stepper.close()
