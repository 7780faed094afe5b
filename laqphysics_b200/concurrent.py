"""Instances of different operators (uneven radial grids, channel sets, fields) stepped at
the same time on one GPU.

Same-operator instances batch into one launch per kernel (torch_backend.step_batched).
Instances whose operators differ cannot share a launch: each keeps its own operator handle,
Krylov workspace and CUDA stream, and a host thread per instance enqueues its step (the
C-ABI calls release the interpreter lock), so the kernels of small, latency-bound solves
run side by side on the SMs instead of one after another.  Every instance gets exactly the
result of stepping it alone (torch_backend.step, including the reference's dt halving).
"""
from concurrent.futures import ThreadPoolExecutor

import torch

from .torch_backend import step


class ConcurrentStepper:
    """schedules: one FieldSchedule per instance, each over its own engine (operator)."""

    def __init__(self, schedules, device='cuda:0'):
        engines = [s.engine for s in schedules]
        if len({id(e) for e in engines}) != len(engines):
            raise ValueError('concurrent instances need one engine each (instances of one operator: step_batched)')
        self.device = torch.device(device)
        self.schedules = list(schedules)
        self.streams = [torch.cuda.Stream(self.device) for _ in self.schedules]
        self.pool = ThreadPoolExecutor(max_workers=len(self.schedules))

    def map(self, fn):
        """fn(i) -> (state, info) for every instance i, each on its own stream and host
        thread; returns ([states], [infos]) once every stream's work is ordered before the
        caller's stream."""
        current = torch.cuda.current_stream(self.device)

        def run(i):
            stream = self.streams[i]
            with torch.cuda.device(self.device):
                stream.wait_stream(current)
                with torch.cuda.stream(stream):
                    y, info = fn(i)
                y.record_stream(current)
            return y, info

        results = list(self.pool.map(run, range(len(self.schedules))))
        for stream in self.streams:
            current.wait_stream(stream)
        return [r[0] for r in results], [r[1] for r in results]

    def step(self, states, t, dt, tol=1e-10, maxdim=48):
        """One midpoint Arnoldi step of every instance from time t; returns (states, infos)."""
        if len(states) != len(self.schedules):
            raise ValueError('one state per instance')
        return self.map(lambda i: step(self.schedules[i], states[i], t, dt, tol, maxdim))

    def cf4(self, states, avecs, t, dt, reference_energies, tol=1e-11):
        """One CF4 Magnus + Pade/GMRES step of every instance (implicit.cf4_step with each
        engine's own preconditioner, field and reference energy)."""
        from .implicit import cf4_step
        if not len(states) == len(avecs) == len(reference_energies) == len(self.schedules):
            raise ValueError('one state, field and reference energy per instance')
        return self.map(lambda i: cf4_step(self.schedules[i].engine, states[i], avecs[i], t, dt,
                                           reference_energies[i], tol))

    def close(self):
        self.pool.shutdown()
