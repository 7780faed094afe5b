"""Instantaneous ionic contraction of the surface flux on the device.

Restates the set-up of the reference's ``SurfaceContractor`` (python/surface_contract.py:5-39)
— active channels, sorted outer (l, m) states, the coupled-basis "fast" path with
Clebsch-Gordan coefficients and the folded-m masks — as one entry list per label:
(frame column, inner ionic state, real coefficient, outer state).  ``__call__`` then
computes q[label, outer, s] = sum_entries coef sum_r conj(chi[inner, r, column]) frame(r, s, col)
in one device launch (python/surface_contract.py:41-56).  Sparse (bipolar) transforms
contribute one entry per non-zero, as the reference's sparse path does.
"""
import ctypes as ct

import numpy as np
import torch
from scipy.sparse import issparse

from ._lib import LIB, check


class SurfaceContractor:
    def __init__(self, h, ion, labels, unique, columns, folded, angular_transform=None, device='cuda:0'):
        self.h, self.ion, self.labels, self.unique, self.columns, self.folded = h, ion, labels, unique, columns, folded
        self.device = torch.device(device)
        key = lambda lm: (lm[0], abs(lm[1]) if folded else lm[1])
        active = [c for c, (inner, outer) in enumerate(h.ch) if key(inner) in ion.index]
        self.outerstates = sorted({h.ch[c][1] for c in active})
        outerindex = {x: i for i, x in enumerate(self.outerstates)}
        self.shape = (len(labels), len(self.outerstates), len(h.surface_indices))
        sparse = angular_transform is not None and issparse(angular_transform)
        if sparse:   # bipolar transforms: every non-zero becomes an entry (python/surface_contract.py:29-32)
            angular_transform = angular_transform.toarray()
        self.transform = angular_transform
        self.fast = bool(angular_transform is not None and folded and not sparse)
        entries = [[] for _ in labels]          # (frame column, inner, coef, outer)
        if self.fast:
            U = angular_transform
            lookup = {pair: i for i, pair in enumerate(h.ch)}
            pairs = []
            for c in range(U.shape[1]):
                support = np.flatnonzero(abs(U[:, c]) > 1e-14)
                pair = {(h.ch[i][0][0], h.ch[i][1][0]) for i in support}
                if len(pair) != 1:
                    raise ValueError('coupled column has no unique radial angular pair')
                pairs.append(next(iter(pair)))
            for j, (n, l, m) in enumerate(labels):
                for c, (l1, l2) in enumerate(pairs):
                    pair = ((l1, m), (l2, -m))
                    if pair in lookup:
                        entries[j].append((c, ion.index[(l1, abs(m) if folded else m)], float(U[lookup[pair], c]),
                                           outerindex[(l2, -m)]))
        else:
            for j, label in enumerate(labels):
                for c in active:
                    (li, mi), outer = h.ch[c]
                    weight = 1.0
                    if folded and mi != label[2]:
                        continue
                    inner = ion.index[key((li, mi))]
                    if angular_transform is None:
                        entries[j].append((c, inner, weight, outerindex[outer]))
                    else:
                        for cc in np.flatnonzero(abs(angular_transform[c]) > 0):
                            entries[j].append((int(cc), inner, float(angular_transform[c, cc]), outerindex[outer]))
        flat = [e for row in entries for e in row]
        self.entry_count = len(flat)
        ptr = np.cumsum([0] + [len(row) for row in entries]).astype(np.int32)
        as_dev = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a, dtype=dt), device=self.device)
        self._eptr = as_dev(ptr, np.int32)
        self._ecol = as_dev([e[0] for e in flat] or [0], np.int32)
        self._einner = as_dev([e[1] for e in flat] or [0], np.int32)
        self._ecoef = as_dev([e[2] for e in flat] or [0.], np.float64)
        self._eouter = as_dev([e[3] for e in flat] or [0], np.int32)
        self._column = as_dev(columns, np.int32)

    @torch.no_grad()
    def contract(self, chi, frame):
        """q on the device.  chi: ((na n), nunique) complex128 (torch, C order); frame: (n, ns, nc)
        complex128 torch tensor of any strides."""
        nlab, nouter, ns = self.shape
        q = torch.empty(self.shape, dtype=torch.complex128, device=self.device)
        chi = chi.contiguous()
        fr, fs, fc = frame.stride()
        stream = ct.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        vp = lambda t: ct.c_void_p(t.data_ptr())
        check(LIB.he_surface_contract(self.h.n, len(self.unique), nlab, nouter, ns, vp(chi), vp(frame), fr, fs, fc,
                                      vp(self._eptr), vp(self._ecol), vp(self._einner), vp(self._ecoef),
                                      vp(self._eouter), vp(self._column), vp(q), stream), 'he_surface_contract')
        return q

    def __call__(self, chi, frame):
        """Reference-compatible call: numpy in, numpy out (the work runs on the device)."""
        as_t = lambda a: a if torch.is_tensor(a) else torch.as_tensor(np.asarray(a, dtype=complex), device=self.device)
        q = self.contract(as_t(chi), as_t(frame))
        return q if torch.is_tensor(frame) else q.cpu().numpy()
