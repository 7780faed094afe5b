"""Device tSURFF flux frames (python/helium3d.py:52-77, python/torch_backend.py:133-138).

The commutator rows surface_T / surface_P are dense only on the few elements that
touch the surface radius; the device keeps just that column window.
"""
import ctypes as ct

import numpy as np
import torch

from ._lib import LIB, check, ptr


class SurfaceFlux:
    def __init__(self, engine):
        h = engine.h
        self.engine = engine
        self.indices = np.asarray(h.surface_indices)
        T = np.asarray(h.surface_T, dtype=complex)
        P = np.asarray(h.surface_P, dtype=complex)
        cols = np.flatnonzero(np.max(np.abs(T), axis=0) + np.max(np.abs(P), axis=0) > 0)
        if not len(cols):
            raise ValueError('empty surface stencil')
        self.lo = int(cols[0])
        self.width = int(cols[-1] - cols[0] + 1)
        self.ns = T.shape[0]
        window = slice(self.lo, self.lo + self.width)
        device = engine.device
        self.J = torch.as_tensor(np.ascontiguousarray(T[:, window]), device=device)
        self.JP = torch.as_tensor(np.ascontiguousarray(P[:, window]), device=device)

    @torch.no_grad()
    def frame(self, x, field):
        """Device tensor (n, ns, nc) (a permuted view of Fortran-ordered storage)."""
        e = self.engine
        e._check(x, torch.complex128)
        out = torch.empty((e.nc, self.ns, e.n), dtype=torch.complex128, device=e.device)
        f = np.ascontiguousarray(field, dtype=np.float64)
        stream = ct.c_void_p(torch.cuda.current_stream(e.device).cuda_stream)
        check(LIB.he_flux(e.op.handle, ct.c_void_p(x.data_ptr()), ct.c_void_p(out.data_ptr()), self.ns, self.lo,
                          self.width, ct.c_void_p(self.J.data_ptr()), ct.c_void_p(self.JP.data_ptr()), ptr(f),
                          stream), 'he_flux')
        return out.permute(2, 1, 0)
