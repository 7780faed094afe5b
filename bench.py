"""Benchmark of the B200 helium engine (one JSON line on stdout from rank 0).

Step = one two-electron H·psi application on the H·psi microbenchmark grid (coupled
l1,l2<=5, L<=3, M=0: nc=43; 60 FE elements of order 9 + 20-point ECS tail: n=560;
N=13,484,800 amplitudes), length gauge, z field 0.02 a.u., complex128 arithmetic.
`value` = H·psi GB/s = algorithmic bytes (read psi + write H·psi = 2 N 16 B) per
application / device time, summed over ranks.  The complex64 mode, the end-to-end
host-buffer figure, the roofline of the kernel and the CPU oracle baseline are
reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU runs are independent replicas (one instance per GPU, no collective on
the data path); timing is the max over ranks of CUDA-event time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = 'H·ψ HBM GB/s (3D He steps/s & H·ψ HBM GB/s: FP64 vs mixed/batched at ≤1e-6 spectrum err)'
WORKLOAD = 'H·ψ microbenchmark: coupled l1,l2<=5 L<=3 M=0 (nc=43), 60 FE x order 9 + 20-pt ECS tail (n=560), N=13.48M'
L2_BYTES = 126 * 2 ** 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=200)
    p.add_argument('--warmup', type=int, default=5)
    p.add_argument('--impl', choices=['b200', 'reference'], default='b200')
    p.add_argument('--no-cpu-baseline', action='store_true')
    p.add_argument('--no-arnoldi', action='store_true', help='skip the Arnoldi steps/s leg')
    p.add_argument('--cfg2-steps', type=int, default=4,
                   help='steps of the mixed-precision config slice on the microbenchmark grid (0: skip)')
    p.add_argument('--path', type=int, default=1, choices=[0, 1, 2, 3],
                   help='H·psi kernel path of the microbenchmark operator (he_set_path; 1 = default fused kernels)')
    p.add_argument('--adjoint-steps', type=int, default=2048, help='adjoint leg: Arnoldi steps (dt 0.005)')
    p.add_argument('--adjoint-knots', type=int, default=512, help='adjoint leg: field samples')
    p.add_argument('--adjoint-checkpoint', type=int, default=None,
                   help='adjoint leg: steps between kept states (default: every state resident in HBM)')
    p.add_argument('--profile', choices=['c128', 'c64', 'arnoldi', 'arnoldi-split', 'batched', 'batched-attempt', 'cf4', 'cfg2',
                                         'pump-probe', 'preconditioner', 'spectrum',
                                         'adjoint', 'concurrent'],
                   default=None,
                   help='run only W+K applications of one precision (for ncu captures); prints no JSON')
    return p.parse_args()


def peaks():
    path = REPO / 'MEASURED_PEAKS.json'
    if path.exists():
        data = json.loads(path.read_text())
        return float(data['hbm_gbs']), float(data['bf16_tflops']), 'measured'
    return 6650.0, 1590.0, 'fallback'


def profile_traffic(name):
    """dram bytes per launch recorded in a committed ncu summary (profiles/<name>.md)."""
    path = REPO / 'profiles' / f'{name}.md'
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        if line.strip().startswith('traffic_bytes_per_launch:'):
            try:
                return float(line.split(':', 1)[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML (read-only queries) every
    millisecond while the timed region runs; falls back to nvidia-smi polling."""
    REASONS = {'hw_slowdown': 0x8, 'hw_thermal_slowdown': 0x40, 'sw_thermal_slowdown': 0x20, 'sw_power_cap': 0x4}

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.samples, self.reason_bits, self.max_mhz = [], 0, None
        self.stop = threading.Event()
        self.nvml = None
        try:
            import pynvml
            pynvml.nvmlInit()
            if isinstance(gpu_id, str) and gpu_id.startswith('GPU-'):
                self.handle = pynvml.nvmlDeviceGetHandleByUUID(gpu_id)
            else:
                self.handle = pynvml.nvmlDeviceGetHandleByIndex(int(gpu_id))
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
            self.nvml = pynvml
        except Exception:
            self.nvml = None

    def __enter__(self):
        self.stop.clear()
        self.thread = threading.Thread(target=self._poll if self.nvml else self._smi, daemon=True)
        self.thread.start()
        return self

    def _poll(self):
        nv = self.nvml
        while not self.stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)))
                self.reason_bits |= int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle))
            except Exception:
                return
            time.sleep(0.001)

    def _smi(self):
        query = 'clocks.sm,clocks.max.sm,clocks_event_reasons.active'
        while not self.stop.is_set():
            try:
                out = subprocess.run(['nvidia-smi', '-i', str(self.gpu_id), f'--query-gpu={query}',
                                      '--format=csv,noheader,nounits'], capture_output=True, text=True, timeout=5)
                sm, mx, active = [x.strip() for x in out.stdout.split(',')[:3]]
                self.samples.append(float(sm))
                self.max_mhz = float(mx)
                self.reason_bits |= int(active, 16) if active.startswith('0x') else 0
            except Exception:
                return

    def __exit__(self, *exc):
        self.stop.set()
        self.thread.join(timeout=5)

    def summary(self):
        reasons = sorted(name for name, bit in self.REASONS.items() if self.reason_bits & bit)
        return {'sm_mhz': float(np.median(self.samples)) if self.samples else None, 'sm_max_mhz': self.max_mhz,
                'samples': len(self.samples), 'reasons': reasons, 'source': 'nvml' if self.nvml else 'nvidia-smi'}


def gpu_identifier(torch, device):
    props = torch.cuda.get_device_properties(device)
    uuid = getattr(props, 'uuid', None)
    if uuid is not None:
        text = str(uuid)
        return text if text.startswith('GPU-') else 'GPU-' + text
    visible = os.environ.get('CUDA_VISIBLE_DEVICES')
    return visible.split(',')[device.index or 0] if visible else device.index or 0


def cpu_oracle_rate(h, psi, field, budget_s):
    """Oracle (C/OpenMP restatement of kernels.f90:119-176) on a bounded channel sample.
    Returns (GB/s of the full-operator equivalent, threads, sample description)."""
    from oracle import cpu
    tables = cpu.host_tables(h)
    start = time.perf_counter()
    cpu.tensor_apply(h, psi, field, False, channels=(0, 1), tables=tables)
    per_channel = max(time.perf_counter() - start, 1e-6)
    count = int(min(h.nc, max(1, budget_s / per_channel)))
    reps = max(1, int(budget_s / (per_channel * count)))
    start = time.perf_counter()
    for _ in range(reps):
        cpu.tensor_apply(h, psi, field, False, channels=(0, count), tables=tables)
    elapsed = time.perf_counter() - start
    gbs = reps * 2 * h.size * 16 * (count / h.nc) / elapsed / 1e9
    sample = (f'{reps} x H.psi over output channels 0..{count - 1} of {h.nc} '
              f'({count / h.nc:.3f} of the state each), complex128, {elapsed:.1f} s')
    return gbs, cpu.threads(), sample


def arnoldi_leg(torch, device, steps, cpu_steps):
    """Plain FP64 Arnoldi propagation (the reference's propagate.step driven as in
    run3d.py:196-199, length gauge, field E(t) along z): 15 elements x order 8 + 12-point
    ECS tail (n=132), coupled l<=3 L<=2 (nc=17), ground-state start, maxdim 12, dt 0.02,
    sin^2 pulse omega 1.6, 10 cycles, F0 0.01.  Returns steps/s on the device and of the
    oracle on the host, plus Krylov dimensions."""
    from laqphysics_b200 import workloads
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.torch_backend import FieldSchedule, step
    h, hreal = workloads.arnoldi_small(), workloads.arnoldi_small_real()
    t_ground = time.perf_counter()
    E0, g, _ = hreal.ground(tol=1e-9)                    # device LOBPCG (laqphysics_b200.ground_s)
    t_ground = time.perf_counter() - t_ground
    ratio = np.sqrt(h.grid.weights / hreal.grid.weights)
    psi0 = (g.reshape(h.shape, order='F') * ratio[:, None, None] * ratio[None, :, None]).ravel(order='F')
    engine = B200Hamiltonian(h, device)
    pulse = workloads.length_pulse()
    field = lambda t: (0., 0., float(pulse.electric(t)))
    apply_at = FieldSchedule(engine, field, velocity=False)
    dt, tol, maxdim = .02, 1e-10, 12
    state = engine.state(psi0)
    for i in range(3):
        state, _ = step(apply_at, state, i * dt, dt, tol, maxdim)
    torch.cuda.synchronize(device)
    dims = []
    applies0 = engine.apply_count
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    t0 = time.perf_counter()
    for i in range(3, 3 + steps):
        state, info = step(apply_at, state, i * dt, dt, tol, maxdim)
        dims.append(info['dimension'])
    stop.record()
    torch.cuda.synchronize(device)
    ms = start.elapsed_time(stop)
    out = {'workload': 'Arnoldi FP64 length gauge: n=132 nc=17 (N=296,208), maxdim 12, dt 0.02, ground-state start',
           'steps': steps, 'steps_per_s': steps / (ms * 1e-3), 'ms_per_step': ms / steps,
           'mean_dimension': float(np.mean(dims)), 'ground_energy': E0, 'ground_state_s': t_ground,
           'hpsi_per_step': (engine.apply_count - applies0) / steps}
    if cpu_steps:
        from oracle import arnoldi, cpu
        from threadpoolctl import threadpool_limits
        x = psi0.copy()
        tables = cpu.host_tables(h)
        # the reference's recommended threading: OpenMP over all cores in H·psi, BLAS on one
        # thread (two thread pools spinning on the same cores slow this loop ~40x)
        with threadpool_limits(limits=1, user_api='blas'):
            t0 = time.perf_counter()
            for i in range(cpu_steps):
                x, _ = arnoldi.step(lambda t, y: cpu.tensor_apply(h, y, field(t), False, tables=tables), x, i * dt, dt,
                                    tol, maxdim)
            el = time.perf_counter() - t0
        out['cpu_baseline'] = {'steps_per_s': cpu_steps / el, 'cores': cpu.threads(), 'kind': 'port',
                               'sample': f'{cpu_steps} Arnoldi steps (oracle numpy Arnoldi + C tensor_apply)'}
    return out


def batched_leg(torch, device, steps, count=32):
    """Batched Arnoldi on the Arnoldi grid (n=132, nc=17): `count` pump-probe-like instances
    (seeded peak fields 0.005-0.03 a.u., delays inside the 10-cycle pulse) stepped together
    by he_expv_batched, in complex128 and in mixed precision (complex64 H·psi inside the
    complex128 Krylov).  Reports instance-steps/s and the mixed-vs-FP64 state difference."""
    from laqphysics_b200 import workloads
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.torch_backend import step_batched
    h, hreal = workloads.arnoldi_small(), workloads.arnoldi_small_real()
    t_ground = time.perf_counter()
    E0, g, _ = hreal.ground(tol=1e-9)                    # device LOBPCG (laqphysics_b200.ground_s)
    t_ground = time.perf_counter() - t_ground
    ratio = np.sqrt(h.grid.weights / hreal.grid.weights)
    psi0 = (g.reshape(h.shape, order='F') * ratio[:, None, None] * ratio[None, :, None]).ravel(order='F')
    engine = B200Hamiltonian(h, device)
    pulse = workloads.length_pulse()
    rng = np.random.default_rng(2026)
    peaks = rng.uniform(.005, .03, count)
    delays = rng.uniform(0., 30., count)
    scale = peaks / .01   # length_pulse has peak 0.01

    def fields_at(t):
        f = np.zeros((count, 3))
        f[:, 2] = scale * np.array([pulse.electric(t + d) for d in delays])
        return f

    dt, tol, maxdim = .02, 1e-10, 12
    x0 = engine.state(psi0).repeat(count).reshape(count, -1).contiguous()
    out = {'workload': f'{count} instances, Arnoldi grid n=132 nc=17, length gauge, maxdim 12, dt 0.02',
           'count': count, 'steps': steps}
    finals = {}
    warm = None
    for precision in ('complex128', 'mixed'):
        x = x0.clone()
        for i in range(3):
            x, _ = step_batched(engine, fields_at, x, i * dt, dt, tol, maxdim, precision=precision)
        if precision == 'complex128':
            warm = x.clone()
        torch.cuda.synchronize(device)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        dims = []
        applies0 = engine.apply_count
        start.record()
        for i in range(3, 3 + steps):
            x, info = step_batched(engine, fields_at, x, i * dt, dt, tol, maxdim, precision=precision)
            dims.append(float(np.mean(info['dimension'])))
        stop.record()
        torch.cuda.synchronize(device)
        ms = start.elapsed_time(stop)
        finals[precision] = x
        out[precision] = {'instance_steps_per_s': count * steps / (ms * 1e-3), 'ms_per_step': ms / steps,
                          'mean_dimension': float(np.mean(dims)),
                          'hpsi_per_instance_step': (engine.apply_count - applies0) / (count * steps)}
    # like for like: the same instances over the same steps (3 .. 3+steps, from the same
    # complex128 states), stepped one at a time by the plain FP64 engine
    from laqphysics_b200.torch_backend import FieldSchedule, step
    torch.cuda.synchronize(device)
    applies0 = engine.apply_count
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    singles = []
    for b in range(count):
        schedule = FieldSchedule(engine, lambda t, b=b: fields_at(t)[b], velocity=False)
        xb = warm[b].contiguous()
        for i in range(3, 3 + steps):
            xb, _ = step(schedule, xb, i * dt, dt, tol, maxdim)
        singles.append(xb)
    stop.record()
    torch.cuda.synchronize(device)
    out['single_fp64_same_instances'] = {
        'instance_steps_per_s': count * steps / (start.elapsed_time(stop) * 1e-3), 'steps_per_instance': steps,
        'hpsi_per_instance_step': (engine.apply_count - applies0) / (count * steps),
        'rel_l2_vs_batched_complex128': float(torch.max(torch.linalg.vector_norm(torch.stack(singles) - finals['complex128'], dim=1)
                                                        / torch.linalg.vector_norm(finals['complex128'], dim=1)))}
    for precision in ('complex128', 'mixed'):
        out[precision]['speedup_vs_single_fp64_same_instances'] = (
            out[precision]['instance_steps_per_s'] / out['single_fp64_same_instances']['instance_steps_per_s'])
    diff = torch.linalg.vector_norm(finals['mixed'] - finals['complex128'], dim=1)
    ref = torch.linalg.vector_norm(finals['complex128'], dim=1)
    out['mixed_vs_fp64_rel_l2_max'] = float((diff / ref).max())
    out['mixed_norm_error_max'] = float((torch.linalg.vector_norm(finals['mixed'], dim=1) - ref).abs().max())
    return out


def adjoint_leg(torch, device, steps=128, knots=32, checkpoint=None):
    """Adjoint gradient on the Arnoldi grid widened to l <= 4: `steps` fixed Arnoldi steps
    (dt 0.005, Krylov tolerance 1e-12, maxdim 30) under a field of `knots` seeded samples
    (two pulses, peak 0.02 a.u.); objective = He+(n = 2) channel yield with the second
    electron beyond 5 a.u. (adjoint.ChannelYield).
    Reports the forward and backward times and their ratio with every state resident (the
    default) and with states kept every 64 steps (segments recomputed).  The defaults are the
    adjoint configuration's stated size: 2048 steps, 512 field samples, checkpoint 64."""
    from laqphysics_b200 import workloads
    from laqphysics_b200.adjoint import Propagation, check_complex_symmetric
    from laqphysics_b200.engine import B200Hamiltonian
    h, hreal = workloads.adjoint_grid(), workloads.adjoint_grid(ecs_angle=0.)
    _, g, _ = hreal.ground(tol=1e-9)
    ratio = np.sqrt(h.grid.weights / hreal.grid.weights)
    psi0 = (g.reshape(h.shape, order='F') * ratio[:, None, None] * ratio[None, :, None]).ravel(order='F')
    engine = B200Hamiltonian(h, device)
    check_complex_symmetric(engine)
    from laqphysics_b200.adjoint import ChannelYield
    objective = ChannelYield(h, device, shell=2, radius=5.)
    dt = .005
    rng = np.random.default_rng(512)
    t = np.linspace(0, steps * dt, knots)
    theta = .02 * (np.exp(-((t - .3 * t[-1]) / (.1 * t[-1])) ** 2) + np.exp(-((t - .7 * t[-1]) / (.1 * t[-1])) ** 2))
    theta *= rng.uniform(.8, 1.2, knots)

    def run(every):
        prop = Propagation(engine, psi0, dt, steps, t, objective, tol=1e-12, maxdim=30, checkpoint=every)
        prop.forward(theta)                               # warm-up (generated kernels, workspaces, graphs)
        prop.gradient()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        J = prop.forward(theta)
        torch.cuda.synchronize(device)
        t1 = time.perf_counter()
        grad = prop.gradient()
        torch.cuda.synchronize(device)
        t2 = time.perf_counter()
        return prop, J, grad, t1 - t0, t2 - t1

    prop, J, grad, fwd, bwd = run(checkpoint)
    _, _, grad32, fwd32, bwd32 = run(64)
    return {'workload': f'adjoint gradient: l1,l2<=4 L<=2 (nc={h.nc}, n={h.n}), {steps} Arnoldi steps dt 0.005, '
                        f'{knots} field samples, objective: He+(n=2) yield, second electron beyond 5 a.u.',
            'checkpoint': prop.checkpoint, 'objective': J, 'forward_ms': fwd * 1e3, 'backward_ms': bwd * 1e3,
            'backward_over_forward': bwd / fwd, 'gradient_norm': float(np.linalg.norm(grad)),
            'checkpoint_64': {'forward_ms': fwd32 * 1e3, 'backward_ms': bwd32 * 1e3,
                              'backward_over_forward': bwd32 / fwd32,
                              'gradient_rel_diff': float(np.linalg.norm(grad32 - grad) / np.linalg.norm(grad))}}


def concurrent_leg(torch, device, count=8, steps=3):
    """Instances of different operators (Arnoldi-type grids with 8-15 tail points, l <= 2
    or 3, L <= 2; own fields) stepped together by laqphysics_b200.concurrent (one stream and
    host thread each) against the same instances stepped one after another; maxdim 12,
    dt 0.02, tol 1e-10, seeded states.  Wall time around synchronized regions."""
    from laqphysics_b200.concurrent import ConcurrentStepper
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.torch_backend import FieldSchedule, step
    from laqphysics_b200 import workloads
    schedules, states, sizes = [], [], []
    for k in range(count):
        h = workloads.coupled(np.linspace(0, 25, 16), 8, 2 + k % 2, 2, ecs_angle=.3, tail=8 + k, cutoff_radii=(18., 22.))
        e = B200Hamiltonian(h, device)
        amp = .005 + .003 * k
        schedules.append(FieldSchedule(e, lambda t, a=amp: (0., 0., a * np.sin(1.6 * t)), velocity=False))
        x = workloads.seeded_state(h.size, 90 + k)
        states.append(e.state(x / np.linalg.norm(x)))
        sizes.append(h.size)
    stepper = ConcurrentStepper(schedules, device)
    dt, tol, maxdim = .02, 1e-10, 12
    stepper.step(states, 0., dt, tol, maxdim)            # warm-up (generated kernels, workspaces)
    for sch, x in zip(schedules, states):
        step(sch, x, 0., dt, tol, maxdim)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    xs = states
    for i in range(steps):
        xs, _ = stepper.step(xs, (i + 1) * dt, dt, tol, maxdim)
    torch.cuda.synchronize(device)
    together = time.perf_counter() - t0
    t0 = time.perf_counter()
    for sch, x in zip(schedules, states):
        for i in range(steps):
            x, _ = step(sch, x, (i + 1) * dt, dt, tol, maxdim)
    torch.cuda.synchronize(device)
    alone = time.perf_counter() - t0
    out = {'workload': f'{count} instances of different operators (N = {min(sizes)}..{max(sizes)}), {steps} Arnoldi '
                       f'steps each, maxdim 12, dt 0.02', 'instance_steps_per_s': count * steps / together,
           'one_after_another_instance_steps_per_s': count * steps / alone, 'speedup': alone / together}
    # the same instances under CF4 + Pade/GMRES steps (velocity gauge, dt 0.05, each with its
    # own separable preconditioner in complex64 and its own pulse)
    from laqphysics_b200.implicit import SeparablePreconditioner, cf4_step
    avecs = [lambda t, a=.01 + .003 * k: np.array([0., 0., a * np.cos(1.6 * t)]) for k in range(count)]
    for sch in schedules:
        sch.engine.separable = SeparablePreconditioner(sch.engine, 'complex64')
    e_ref = [-2.9] * count
    xs, _ = stepper.cf4(states, avecs, 0., .05, e_ref, 1e-10)            # warm-up
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for i in range(steps):
        xs, _ = stepper.cf4(xs, avecs, (i + 1) * .05, .05, e_ref, 1e-10)
    torch.cuda.synchronize(device)
    together = time.perf_counter() - t0
    t0 = time.perf_counter()
    for sch, av, x in zip(schedules, avecs, states):
        for i in range(steps):
            x, _ = cf4_step(sch.engine, x, av, (i + 1) * .05, .05, -2.9, 1e-10)
    torch.cuda.synchronize(device)
    alone = time.perf_counter() - t0
    stepper.close()
    out['cf4'] = {'workload': f'the same instances, {steps} CF4 + Pade/GMRES steps each (dt 0.05, complex64 '
                              f'separable preconditioners)', 'instance_steps_per_s': count * steps / together,
                  'one_after_another_instance_steps_per_s': count * steps / alone, 'speedup': alone / together}
    return out


def pump_probe_leg(torch, device, count=32, steps=2):
    """The batched pump-probe configuration's shape at a size that fits one GPU for 32
    instances at once: bipolar all-M channels (l1, l2 <= 3 or 4 alternating, total L <= 1),
    10 or 12 finite elements of order 9 on [0, 25] a.u. + 8-point ECS tail, circular (sigma+)
    probe pulses (omega 1.6 a.u., 6 cycles) with seeded delays 0-800 a.u. and peak fields
    0.005-0.03 a.u., CF4 + Pade/GMRES steps dt 0.05 (tol 1e-10) from the ground state, in the
    middle of each instance's probe.  The stated 40-60 elements x order 10 with l <= 6 and
    every total L would need up to 2.4 GB per state and ~78 GB of FGMRES basis per instance.
    Three ways: the plain FP64 engine (complex128 preconditioner, GMRES(32)) one instance
    after another; complex64 preconditioners (FGMRES(16)) one after another; and all 32
    instances stepped together (laqphysics_b200.concurrent: own engine, stream and host thread
    each, complex64 preconditioners)."""
    from dataclasses import replace
    from laqphysics_b200.bipolar import BipolarHelium
    from laqphysics_b200.concurrent import ConcurrentStepper
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.fedvr import make_grid
    from laqphysics_b200.implicit import SeparablePreconditioner, cf4_step
    from laqphysics_b200.pulses import Pulse
    from laqphysics_b200.torch_backend import FieldSchedule
    shapes = {}
    for lmax, elements in ((3, 10), (4, 12)):
        grid = lambda angle: make_grid(np.linspace(0, 25, elements + 1), 9, ecs_angle=angle, tail=8)
        h = BipolarHelium(grid(.3), lmax=lmax, total_Lmax=1, M=None, cutoff_radii=(18., 22.))
        hreal = BipolarHelium(grid(0.), lmax=lmax, total_Lmax=1, M=None, cutoff_radii=(18., 22.))
        E0, g, _ = hreal.ground(tol=1e-9)
        ratio = np.sqrt(h.grid.weights / hreal.grid.weights)
        psi0 = (g.reshape(h.shape, order='F') * ratio[:, None, None] * ratio[None, :, None]).ravel(order='F')
        shapes[lmax] = (h, psi0, E0)
    rng = np.random.default_rng(33)
    delays, peaks = rng.uniform(0, 800, count), rng.uniform(.005, .03, count)
    probe = Pulse(omega=1.6, cycles=6, field=1.)
    avecs, engines, states, e_ref, sizes = [], [], [], [], []
    for k in range(count):
        h, psi0, E0 = shapes[3 + k % 2]
        pk = replace(probe, field=float(peaks[k]), start=float(delays[k]))
        skew = replace(pk, cep=pk.cep - np.pi / 2)
        t_mid = delays[k] + probe.duration / 2
        avecs.append(lambda t, pk=pk, skew=skew, t0=t_mid: np.array([pk.vector(t + t0), skew.vector(t + t0), 0.])
                     / np.sqrt(2))
        engine = B200Hamiltonian(h, device)
        engines.append(engine)
        states.append(engine.state(psi0))
        e_ref.append(E0)
        sizes.append(h.size)
    dt, tol = .05, 1e-10
    out = {'workload': f'{count} bipolar all-M instances (nc = {min(s[0].nc for s in shapes.values())}..'
                       f'{max(s[0].nc for s in shapes.values())}, N = {min(sizes):,}..{max(sizes):,}), sigma+ probes, '
                       f'{steps} CF4 steps each, dt 0.05', 'count': count, 'steps': steps}

    def alone(precision):
        for e in engines:
            e.separable = SeparablePreconditioner(e, precision)
        for e, av, x, er in zip(engines, avecs, states, e_ref):     # warm-up
            cf4_step(e, x, av, 0., dt, er, tol)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        finals = []
        for e, av, x, er in zip(engines, avecs, states, e_ref):
            for i in range(steps):
                x, _ = cf4_step(e, x, av, i * dt, dt, er, tol)
            finals.append(x)
        torch.cuda.synchronize(device)
        return count * steps / (time.perf_counter() - t0), finals

    fp64, ref = alone('complex128')
    c64, _ = alone('complex64')
    stepper = ConcurrentStepper([FieldSchedule(e, av, velocity=True) for e, av in zip(engines, avecs)], device)
    stepper.cf4(states, avecs, 0., dt, e_ref, tol)                  # warm-up
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    xs = states
    for i in range(steps):
        xs, _ = stepper.cf4(xs, avecs, i * dt, dt, e_ref, tol)
    torch.cuda.synchronize(device)
    together = count * steps / (time.perf_counter() - t0)
    stepper.close()
    err = max(float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)) for a, b in zip(xs, ref))
    out.update(plain_fp64_one_after_another_instance_steps_per_s=fp64,
               complex64_preconditioner_one_after_another_instance_steps_per_s=c64,
               concurrent_complex64_preconditioner_instance_steps_per_s=together,
               speedup_vs_plain_fp64=together / fp64, state_rel_l2_vs_plain_fp64_max=err)
    return out


def cfg2_slice_leg(torch, device, steps=6):
    """Bounded slice of the mixed-precision full propagation on the microbenchmark grid
    (n = 560, nc = 43, real to 120 a.u.): sin^2 pulse omega 1.6 a.u., 20 cycles, peak
    0.02 a.u., velocity gauge, Arnoldi order 16, dt 0.05, Krylov tolerance 1e-10, tSURFF at
    R_s = 100 a.u. with the He+ n <= 3 channels (6 labels), default energy grid (397) and
    32 polar directions.  `steps` steps from the middle of the pulse (t0 = 39.25 a.u.), started
    from the ground state, a surface sample after every step (channel functions propagated
    back from the slice's end; Volkov phases referenced to t0), in complex128 and in mixed
    precision (complex64 H·psi inside the complex128 Krylov).  Reports steps/s, H·psi per
    step, the slice's spectrum and state errors of the mixed run against the complex128 run,
    and the projection to the full 1571-step run at the measured rates."""
    from laqphysics_b200 import workloads
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.ionic_adjoint import channel_functions
    from laqphysics_b200.pulses import Pulse
    from laqphysics_b200.surface3d import Ionic
    from laqphysics_b200.surface_contract import SurfaceContractor
    from laqphysics_b200.tsurff_run import run, spectrum_error
    h, hreal = workloads.hpsi_microbench(), workloads.hpsi_microbench(ecs_angle=0.)
    base = h.uncoupled
    base.prepare_surface(100.)
    h.prepare_surface(100.)
    labels = [(1, 0, 0), (2, 0, 0), (2, 1, 0), (3, 0, 0), (3, 1, 0), (3, 2, 0)]
    ion = Ionic(base, {0})
    contractor = SurfaceContractor(base, ion, labels, labels, list(range(6)), True, h.transform, device)
    pulse = Pulse(omega=1.6, cycles=20, field=.02)
    avec = lambda t: np.array([0., 0., float(pulse.vector(t))])
    dt = .05
    t0 = round(pulse.duration / 2 / dt) * dt
    t_ground = time.perf_counter()
    _, g, _ = hreal.ground(tol=1e-9)
    t_ground = time.perf_counter() - t_ground
    ratio = np.sqrt(h.grid.weights / hreal.grid.weights)
    psi0 = (g.reshape(h.shape, order='F') * ratio[:, None, None] * ratio[None, :, None]).ravel(order='F')
    chi = channel_functions(ion, labels, avec, t0 + dt * np.arange(steps + 1), device)
    engine = B200Hamiltonian(h, device)
    config = {'M': 0}
    out = {'workload': f'mixed-precision config slice: n={h.n} nc={h.nc} (N={h.size:,}), velocity gauge, Arnoldi order 16, '
                       f'dt 0.05, tol 1e-10, {steps} steps from t0={t0:.2f} a.u. (mid-pulse, 20-cycle sin^2, '
                       f'omega 1.6, 0.02 a.u.), ground-state start, tSURFF at R_s=100 with He+ n<=3 (6 labels)',
           'steps': steps, 'ground_state_s': t_ground}
    results = {}
    for precision in ('complex128', 'mixed'):
        applies = engine.apply_count
        torch.cuda.synchronize(device)
        start = time.perf_counter()
        acc, psi, dim = run(engine, contractor, config, psi0, avec, dt, steps, chi, precision, tol=1e-10, maxdim=16,
                            t0=t0)
        torch.cuda.synchronize(device)
        seconds = time.perf_counter() - start
        results[precision] = (acc, psi)
        out[precision] = {'steps_per_s': steps / seconds, 's_per_step': seconds / steps,
                          'hpsi_per_step': (engine.apply_count - applies) / steps, 'mean_dimension': dim,
                          'full_run_projection_h': 1571 * seconds / steps / 3600}
    rel, per_label = spectrum_error(results['mixed'][0], results['complex128'][0])
    a, b = results['mixed'][1], results['complex128'][1]
    out['spectrum_rel_l2_mixed_vs_fp64'] = rel
    out['angle_integrated_rel_max_mixed_vs_fp64'] = per_label
    out['state_rel_l2_mixed_vs_fp64'] = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
    out['norm_error_mixed_vs_fp64'] = abs(float(torch.linalg.vector_norm(a)) - float(torch.linalg.vector_norm(b)))
    out['mixed_speedup'] = out['mixed']['steps_per_s'] / out['complex128']['steps_per_s']
    return out


def preconditioner_leg(torch, device):
    """The separable preconditioner's GEMM chain on the microbenchmark grid (n = 560, nc = 43,
    l <= 5: 241 GFLOP of complex GEMM per apply, 32 n^3 nc) in both precisions, against the
    same count of torch.bmm calls (cuBLAS Z/CGEMM) on the same box: complex128 on the FP64
    tensor cores (DMMA), complex64 on tcgen05 (TF32, split operands, 3 MMAs per K slice)."""
    from laqphysics_b200 import workloads
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.implicit import SeparablePreconditioner
    h = workloads.hpsi_microbench()
    engine = B200Hamiltonian(h, device)
    x = engine.state(workloads.seeded_state(h.size, 7))
    flops = 32.0 * h.n ** 3 * h.nc
    out = {'workload': f'separable preconditioner, n={h.n} nc={h.nc}: 4 complex n^3 GEMMs per channel + resolvent',
           'gflop_per_apply': flops / 1e9}

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize(device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize(device)
        return a.elapsed_time(b) / reps

    for precision, dtype in (('complex128', torch.complex128), ('complex64', torch.complex64)):
        pre = SeparablePreconditioner(engine, precision)
        ms = timed(lambda: pre.apply(x, .05 / (3 + 1j * np.sqrt(3)), -2.))
        A = torch.randn(h.nc, h.n, h.n, dtype=dtype, device=device)
        B = torch.randn(h.nc, h.n, h.n, dtype=dtype, device=device)
        ref = timed(lambda: [torch.bmm(A, B) for _ in range(4)])
        out[precision] = {'ms_per_apply': ms, 'tflops': flops / (ms * 1e-3) / 1e12,
                          'cublas_bmm_x4_ms': ref, 'cublas_tflops': flops / (ref * 1e-3) / 1e12,
                          'speedup_vs_cublas': ref / ms}
        del pre
    return out


def cf4_leg(torch, device, steps=10):
    """CF4 Magnus steps, each exponential a [2/2] Pade pair of shifted solves by right-
    preconditioned GMRES (the reference's implicit.py:45-109 path), on the Arnoldi grid
    (n=132, nc=17), velocity gauge, sin^2 pulse omega 1.6 a.u. peak 0.02 a.u., dt 0.05,
    ground-state start, reference energy = ground energy, GMRES tolerance 1e-10; separable
    ionic preconditioner in complex128 (GMRES(32)) and in complex64 (flexible GMRES(16)), and
    the mixed form (complex128 defect correction around complex64 inner solves) with the
    state error against the complex128 run.  Also times the preconditioner alone (4 n^3
    complex GEMMs per channel)."""
    from laqphysics_b200 import workloads
    from laqphysics_b200.engine import B200Hamiltonian
    from laqphysics_b200.implicit import SeparablePreconditioner, cf4_step
    from laqphysics_b200.pulses import Pulse
    h, hreal = workloads.arnoldi_small(), workloads.arnoldi_small_real()
    E0, g, _ = hreal.ground(tol=1e-9)
    ratio = np.sqrt(h.grid.weights / hreal.grid.weights)
    psi0 = (g.reshape(h.shape, order='F') * ratio[:, None, None] * ratio[None, :, None]).ravel(order='F')
    engine = B200Hamiltonian(h, device)
    pulse = Pulse(omega=1.6, cycles=10, field=.02)
    avec = lambda t: np.array([0., 0., float(pulse.vector(t))])
    dt, tol = .05, 1e-10
    out = {'workload': 'CF4 + [2/2] Pade / GMRES, Arnoldi grid n=132 nc=17, velocity gauge, dt 0.05, tol 1e-10, '
                       'separable preconditioner', 'steps': steps}
    gemm_flops = 32 * h.n ** 3 * h.nc
    finals = {}
    for variant in ('complex128', 'complex64', 'mixed'):
        precision = 'complex128' if variant == 'complex128' else 'complex64'     # of the preconditioner
        solve = 'mixed' if variant == 'mixed' else 'complex128'                  # of H·psi in the solves
        engine.separable = SeparablePreconditioner(engine, precision)
        x = engine.state(psi0)
        for i in range(2):
            x, _ = cf4_step(engine, x, avec, i * dt, dt, E0, tol=tol, precision=solve)
        torch.cuda.synchronize(device)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        iterations = 0
        start.record()
        for i in range(2, 2 + steps):
            x, info = cf4_step(engine, x, avec, i * dt, dt, E0, tol=tol, precision=solve)
            iterations += info['linear_iterations']
        stop.record()
        finals[variant] = x
        torch.cuda.synchronize(device)
        ms = start.elapsed_time(stop)
        y = x   # complex128 in and out; the complex64 preconditioner converts inside
        for _ in range(3):
            engine.separable.apply(y, dt / 6, .01)
        torch.cuda.synchronize(device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(20):
            engine.separable.apply(y, dt / 6, .01)
        b.record()
        torch.cuda.synchronize(device)
        pre_ms = a.elapsed_time(b) / 20
        out[variant] = {'steps_per_s': steps / (ms * 1e-3), 'ms_per_step': ms / steps,
                        'gmres_iterations_per_step': iterations / steps,
                        'preconditioner_ms': pre_ms, 'preconditioner_tflops': gemm_flops / (pre_ms * 1e-3) / 1e12}
    ref = finals['complex128']
    out['mixed']['solve'] = ('complex128 defect correction around complex64 inner GMRES solves '
                             '(complex64 H·psi, complex64 separable preconditioner)')
    out['mixed']['state_rel_l2_vs_complex128'] = float(torch.linalg.vector_norm(finals['mixed'] - ref) /
                                                       torch.linalg.vector_norm(ref))
    return out


def spectrum_leg(torch, device):
    """Channel-resolved tSURFF on the small case of laqphysics_b200.tsurff_run: complex128
    and mixed-precision propagations with a surface sample every step; spectrum error of
    the mixed run against the complex128 one, and both wall times."""
    from laqphysics_b200.tsurff_run import SMALL_CASE, build_case, run, spectrum_error
    dt = .02
    engine, contractor, psi0, avec, steps, chi = build_case(SMALL_CASE, device, dt)
    run(engine, contractor, SMALL_CASE, psi0, avec, dt, 20, chi, 'complex128')   # warm-up (generated kernels)
    run(engine, contractor, SMALL_CASE, psi0, avec, dt, 20, chi, 'mixed')
    out = {'workload': f'tSURFF small case: n={engine.n} nc={engine.nc}, {steps} velocity-gauge Arnoldi steps '
                       f'dt {dt}, surface sample every step, He+ n<=2 channels'}
    res = {}
    for precision in ('complex128', 'mixed'):
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        res[precision] = run(engine, contractor, SMALL_CASE, psi0, avec, dt, steps, chi, precision)
        torch.cuda.synchronize(device)
        out[precision] = {'steps_per_s': steps / (time.perf_counter() - t0), 'mean_dimension': res[precision][2]}
    # the He+ channel functions of the run: backward CF4 on the device (laqphysics_b200.ionic_adjoint)
    from laqphysics_b200.ionic_adjoint import channel_functions
    from laqphysics_b200.surface3d import Ionic
    ion = Ionic(engine.h.uncoupled, {0})
    unique = [(1, 0, 0), (2, 0, 0), (2, 1, 0)]
    times = dt * np.arange(steps + 1)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    channel_functions(ion, unique, avec, times, device)
    torch.cuda.synchronize(device)
    out['ionic_channel_functions'] = {'frames': steps + 1, 'ms': (time.perf_counter() - t0) * 1e3,
                                      'method': 'backward CF4 + Pade/GMRES (tol 1e-12) on the device'}
    rel, per_label = spectrum_error(res['mixed'][0], res['complex128'][0])
    p64, p32 = res['complex128'][1], res['mixed'][1]
    out['spectrum_rel_l2_mixed_vs_fp64'] = rel
    out['angle_integrated_rel_max_mixed_vs_fp64'] = per_label
    out['state_rel_l2_mixed_vs_fp64'] = float(torch.linalg.vector_norm(p32 - p64) / torch.linalg.vector_norm(p64))
    out['norm_error_mixed_vs_fp64'] = float(abs(torch.linalg.vector_norm(p32) - torch.linalg.vector_norm(p64)))
    out['surface_sample'] = sample_timing(torch, device, engine, contractor, avec, p64, chi)
    return out


def sample_timing(torch, device, engine, contractor, avec, state, chi, count=200):
    """One surface sample (flux frame, contraction, Volkov update) as one launch
    (he_sample_record) and as three (he_flux, he_surface_contract, he_volkov_add): device
    time per sample (CUDA events over `count` samples) and host time per call."""
    from laqphysics_b200.streaming_surface import SurfaceSampler, VolkovAccumulator
    from laqphysics_b200.tsurff_run import SMALL_CASE
    out = {}
    for name, fused in (('one_launch', True), ('three_launches', False)):
        sampler = SurfaceSampler(engine, contractor, VolkovAccumulator(contractor, SMALL_CASE, avec, device=device),
                                 fused=fused)
        for i in range(5):
            sampler.record(i, .02 * i, state, avec(.02 * i), chi[i])
        torch.cuda.synchronize(device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record()
        for i in range(5, 5 + count):
            sampler.record(i, .02 * i, state, avec(.02 * i), chi[i % len(chi)])
        b.record()
        host = (time.perf_counter() - t0) / count
        torch.cuda.synchronize(device)
        out[name] = {'us_per_sample': a.elapsed_time(b) * 1e3 / count, 'host_us_per_call': host * 1e6}
    return out


def run_reference(args, rank):
    """--impl reference: the CPU oracle of the reference's native H·psi on host cores."""
    if rank != 0:
        return 0
    os.environ.setdefault('OMP_NUM_THREADS', str(os.cpu_count()))
    from laqphysics_b200 import workloads
    from oracle import cpu
    h = workloads.hpsi_microbench()
    psi = workloads.seeded_state(h.size, 1234)
    field = (0., 0., .02)
    tables = cpu.host_tables(h)
    start = time.perf_counter()
    cpu.tensor_apply(h, psi, field, False, channels=(0, 1), tables=tables)
    per_channel = max(time.perf_counter() - start, 1e-6)
    budget = 150.0 / max(1, args.steps + args.warmup)
    count = int(min(h.nc, max(1, budget / per_channel)))
    for _ in range(args.warmup):
        cpu.tensor_apply(h, psi, field, False, channels=(0, count), tables=tables)
    start = time.perf_counter()
    for _ in range(args.steps):
        cpu.tensor_apply(h, psi, field, False, channels=(0, count), tables=tables)
    elapsed = time.perf_counter() - start
    frac = count / h.nc
    gbs = 2 * h.size * 16 * frac * args.steps / elapsed / 1e9
    sample = f'each step: output channels 0..{count - 1} of {h.nc} ({frac:.3f} of one H.psi), complex128'
    line = {'impl': 'reference', 'metric': METRIC, 'value': gbs, 'unit': 'GB/s', 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': elapsed / args.steps * 1e3 / frac,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'complex128',
            'data': 'synthetic (seeded complex Gaussian state)',
            'config': {'workload': WORKLOAD, 'field': 'length gauge, Ez=0.02', 'parallelism': 'replicas'},
            'cpu_baseline': {'value': gbs, 'unit': 'GB/s', 'cores': cpu.threads(), 'kind': 'port', 'sample': sample},
            'e2e': {'value': gbs, 'unit': 'GB/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    rank = int(os.environ.get('RANK', 0))
    world = int(os.environ.get('WORLD_SIZE', 1))
    local = int(os.environ.get('LOCAL_RANK', 0))
    if args.impl == 'reference':
        return run_reference(args, rank)
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if world > 1:
        dist.init_process_group('nccl', timeout=timedelta(seconds=300), device_id=torch.device('cuda', local))
    device = torch.device('cuda', local)
    torch.cuda.set_device(device)
    from laqphysics_b200 import workloads
    from laqphysics_b200.engine import B200Hamiltonian

    def barrier():
        if world > 1:
            dist.barrier()

    if args.profile == 'arnoldi':   # W + K Arnoldi steps on the small grid, for launch lists
        arnoldi_leg(torch, device, steps=args.steps, cpu_steps=0)
        return 0
    if args.profile == 'batched':
        print(json.dumps(batched_leg(torch, device, steps=args.steps)), flush=True)
        return 0
    if args.profile == 'cf4':
        print(json.dumps(cf4_leg(torch, device, steps=args.steps)), flush=True)
        return 0
    if args.profile == 'pump-probe':
        print(json.dumps(pump_probe_leg(torch, device)), flush=True)
        return 0
    if args.profile == 'preconditioner':
        print(json.dumps(preconditioner_leg(torch, device)), flush=True)
        return 0
    if args.profile == 'cfg2':
        print(json.dumps(cfg2_slice_leg(torch, device, steps=args.steps)), flush=True)
        return 0
    if args.profile == 'spectrum':
        print(json.dumps(spectrum_leg(torch, device)), flush=True)
        return 0
    if args.profile == 'arnoldi-split':   # CUDA-event cost of one H·psi and of 12-iteration attempts
        from laqphysics_b200 import workloads
        from laqphysics_b200.engine import B200Hamiltonian
        from laqphysics_b200.torch_backend import FieldOperator, exponential_action, step_batched
        h = workloads.arnoldi_small()
        engine = B200Hamiltonian(h, device)
        x = engine.state(workloads.seeded_state(h.size, 1))
        x /= torch.linalg.vector_norm(x)

        def per_call_us(fn, reps):
            for _ in range(3):
                fn()
            torch.cuda.synchronize(device)
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            for _ in range(reps):
                fn()
            stop.record()
            torch.cuda.synchronize(device)
            return start.elapsed_time(stop) / reps * 1e3

        def attempt(count, precision):
            if count == 1:
                op = FieldOperator(engine, (0., 0., .01), velocity=False, precision=precision)
                call = lambda: exponential_action(op, x, .02, 1e-300, 12)
            else:
                xb = x.repeat(count).reshape(count, -1).contiguous()
                fields = np.zeros((count, 3))
                fields[:, 2] = .01
                call = lambda: step_batched(engine, lambda t: fields, xb, 0., .02, 1e-300, 12, precision=precision,
                                            depth=8)

            def run():
                try:
                    call()
                except RuntimeError:   # tol 1e-300: every attempt runs to maxdim and reports non-convergence
                    pass
            return run

        out = {'apply_us': per_call_us(lambda: engine.apply(x, (0., 0., .01), False), 200)}
        for count in (1, 2, 4, 8, 16, 32):
            for precision in ('complex128', 'mixed'):
                out[f'attempt12_us_per_instance_{precision}_x{count}'] = per_call_us(attempt(count, precision), 10) / count
        from laqphysics_b200 import torch_backend
        torch_backend.use_cuda_graphs(False)   # the same solves launched kernel by kernel
        for count in (1, 32):
            out[f'attempt12_us_per_instance_complex128_x{count}_no_graph'] = per_call_us(attempt(count, 'complex128'),
                                                                                        10) / count
        torch_backend.use_cuda_graphs(True)
        print(json.dumps(out), flush=True)
        return 0
    if args.profile == 'batched-attempt':   # two 12-iteration attempts of 32 instances (every one runs to maxdim)
        from laqphysics_b200 import workloads
        from laqphysics_b200.engine import B200Hamiltonian
        from laqphysics_b200.torch_backend import step_batched
        h = workloads.arnoldi_small()
        engine = B200Hamiltonian(h, device)
        x = engine.state(workloads.seeded_state(h.size, 1))
        x /= torch.linalg.vector_norm(x)
        xb = x.repeat(32).reshape(32, -1).contiguous()
        fields = np.zeros((32, 3))
        fields[:, 2] = .01
        for _ in range(2):
            try:
                step_batched(engine, lambda t: fields, xb, 0., .02, 1e-300, 12, depth=8)
            except RuntimeError:
                pass
        torch.cuda.synchronize(device)
        return 0
    if args.profile == 'concurrent':
        print(json.dumps(concurrent_leg(torch, device)), flush=True)
        return 0
    if args.profile == 'adjoint':
        print(json.dumps(adjoint_leg(torch, device, args.adjoint_steps, args.adjoint_knots, args.adjoint_checkpoint)),
              flush=True)
        return 0
    h = workloads.hpsi_microbench()
    engine = B200Hamiltonian(h, device)
    if args.path != 1:
        engine.set_path(args.path)
    field = (0., 0., .02)
    N = h.size
    bytes128 = 2 * N * 16
    inputs = [torch.as_tensor(workloads.seeded_state(N, 1234 + 7 * rank + k), device=device) for k in range(2)]
    out = torch.empty_like(inputs[0])
    in64 = [x.to(torch.complex64) for x in inputs]
    out64 = torch.empty_like(in64[0])
    stream = torch.cuda.current_stream(device)

    def timed(fn, steps):
        barrier()
        torch.cuda.synchronize(device)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for k in range(steps):
            fn(k)
        stop.record(stream)
        torch.cuda.synchronize(device)
        barrier()
        ms = start.elapsed_time(stop)
        if world > 1:
            t = torch.tensor([ms], device=device, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    step128 = lambda k: engine.apply(inputs[k % 2], field, False, out=out)
    step64 = lambda k: engine.apply(in64[k % 2], field, False, out=out64)
    host_in = [torch.empty(N, dtype=torch.complex128).pin_memory() for _ in range(2)]
    for k in range(2):
        host_in[k].copy_(inputs[k].cpu())
    host_out = [torch.empty_like(host_in[0]).pin_memory() for _ in range(2)]
    dev_in = torch.empty_like(inputs[0])

    def step_e2e(k):   # one state at a time: H2D, apply, D2H in sequence
        dev_in.copy_(host_in[k % 2], non_blocking=True)
        engine.apply(dev_in, field, False, out=out)
        host_out[k % 2].copy_(out, non_blocking=True)

    def e2e_stream(count):   # B200Hamiltonian.apply_host_stream: transfers overlapped with compute
        engine.apply_host_stream([host_in[k % 2] for k in range(count)], field, False,
                                 [host_out[k % 2] for k in range(count)])

    if args.profile:
        step = step128 if args.profile == 'c128' else step64
        for k in range(args.warmup + args.steps):
            step(k)
        torch.cuda.synchronize(device)
        return 0
    for k in range(max(3, args.warmup)):
        step128(k); step64(k); step_e2e(k)
    e2e_stream(3)
    torch.cuda.synchronize(device)
    launches0 = engine.apply_count
    with ClockSampler(gpu_identifier(torch, device)) as clocks:
        ms128 = timed(step128, args.steps)
        launches = (engine.apply_count - launches0) * engine.launches_per_apply
        ms64 = timed(step64, args.steps)
        e2e_steps = max(3, min(args.steps, 20))
        ms_e2e_seq = timed(step_e2e, e2e_steps)
        ms_e2e = timed(lambda k: e2e_stream(e2e_steps) if k == 0 else None, 1)
    per128 = ms128 / args.steps
    per64 = ms64 / args.steps
    per_e2e = ms_e2e / e2e_steps
    per_e2e_seq = ms_e2e_seq / e2e_steps
    value = world * bytes128 / (per128 * 1e-3) / 1e9
    value64 = world * (2 * N * 8) / (per64 * 1e-3) / 1e9
    e2e = world * bytes128 / (per_e2e * 1e-3) / 1e9
    hbm, _, peak_kind = peaks()
    flops = workloads.hpsi_flops(h)
    parts = workloads.hpsi_flop_parts(h)
    from laqphysics_b200.engine import fp64_peaks
    fp64 = fp64_peaks(device)
    # compute floor of one apply: kinetic on the FP64 tensor pipe, the rest on the FMA pipe
    floor_ms = (parts['kinetic'] / (fp64['dmma'] * 1e12) + (flops - parts['kinetic']) / (fp64['dfma'] * 1e12)) * 1e3
    achieved = bytes128 / (per128 * 1e-3) / 1e9
    line = {
        'metric': METRIC, 'value': value, 'unit': 'GB/s', 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': per128, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'complex128', 'data': 'synthetic (seeded complex Gaussian state)',
        'config': {'workload': WORKLOAD, 'field': 'length gauge, Ez=0.02', 'parallelism': 'replicas',
                   'l2': 'two rotating 216 MB input states (> 126 MB L2)'},
        'gpu_launches': launches,
        'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': hbm, 'unit': 'GB/s', 'frac': achieved / hbm,
                     'traffic': profile_traffic('hpsi_c128_microbench'), 'peak_kind': peak_kind,
                     'kernel': ' + '.join(engine.kernels()) + ' (one apply)',
                     'plan': engine.plan_info,
                     'fp64_tflops': flops / (per128 * 1e-3) / 1e12, 'flops_per_apply': flops},
        'roofline_fp64': {'bound': 'fp64 (kinetic: DMMA pipe, mixing: DFMA pipe)', 'unit': 'TFLOP/s',
                          'achieved': flops / (per128 * 1e-3) / 1e12, 'peak_dmma': fp64['dmma'],
                          'peak_dfma': fp64['dfma'], 'peak_kind': 'measured in this run (he_fp64_peak)',
                          'flops_per_apply': parts, 'compute_floor_ms': floor_ms, 'frac': floor_ms / per128},
        'complex64': {'value': value64, 'unit': 'GB/s', 'ms_per_step': per64,
                      'frac': value64 / world / hbm, 'speedup_vs_complex128': per128 / per64},
        'e2e': {'value': e2e, 'unit': 'GB/s', 'ms_per_step': per_e2e, 'steps': e2e_steps,
                'h2d_bytes_per_step': N * 16, 'd2h_bytes_per_step': N * 16,
                'path': 'B200Hamiltonian.apply_host_stream over pinned host states: H2D of state k+1 and D2H '
                        'of state k-1 overlap the apply of state k',
                'sequential': {'value': world * bytes128 / (per_e2e_seq * 1e-3) / 1e9, 'ms_per_step': per_e2e_seq,
                               'path': 'pinned host psi -> H2D -> B200Hamiltonian.apply -> D2H, one state at a time'}},
        'clocks': clocks.summary(),
    }
    if not args.no_arnoldi:
        line['arnoldi'] = arnoldi_leg(torch, device, steps=max(10, min(args.steps, 100)),
                                      cpu_steps=0 if (args.no_cpu_baseline or world > 1 or rank) else 3)
        line['batched'] = batched_leg(torch, device, steps=max(5, min(args.steps, 30)))
        line['adjoint'] = adjoint_leg(torch, device, args.adjoint_steps, args.adjoint_knots, args.adjoint_checkpoint)
        line['spectrum'] = spectrum_leg(torch, device)
        line['cf4'] = cf4_leg(torch, device)
        line['preconditioner'] = preconditioner_leg(torch, device)
        line['concurrent'] = concurrent_leg(torch, device)
        line['pump_probe'] = pump_probe_leg(torch, device)
        if args.cfg2_steps:
            line['cfg2_slice'] = cfg2_slice_leg(torch, device, steps=args.cfg2_steps)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        os.environ.setdefault('OMP_NUM_THREADS', str(os.cpu_count()))
        gbs, cores, sample = cpu_oracle_rate(h, workloads.seeded_state(N, 1234), field, 15.0)
        line['cpu_baseline'] = {'value': gbs, 'unit': 'GB/s', 'cores': cores, 'kind': 'port', 'sample': sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == '__main__':
    sys.exit(main())
