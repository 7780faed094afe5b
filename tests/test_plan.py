"""The tiled H·psi plan, checked on the CPU.

The C-ABI exposes the host planner (he_plan_build / he_plan_array, no GPU needed).
A numpy emulation that follows the loops of hpsi_radial_kernel and hpsi_mix_kernel
(tile extents, element blocks, bridge rows, wide edges) must reproduce the oracle
H·psi; every shared-memory extent the kernels use is asserted against its buffer.
"""
import ctypes as ct
import json

import numpy as np
import pytest

from conftest import Tables, golden
from oracle import cpu

RAD_TMAX, RAD_CHUNK, MIX_GROUP, RAD_STRIDE = 40, 8, 4, 41


def build_plan(h):
    from laqphysics_b200 import _lib
    from laqphysics_b200.engine import _host_tables
    t = _host_tables(h)
    p = _lib.ptr
    handle = _lib.LIB.he_plan_build(h.n, h.nc, p(t['ptr']), p(t['col']), p(t['tv']), len(t['vc']), p(t['vptr']),
                                    p(t['vc']), p(t['vl']), p(t['vcoef']), t['nlam'], len(t['dc']), p(t['dptr']),
                                    p(t['dc']), p(t['de']), p(t['r']))
    try:
        def get(which, dtype):
            count = _lib.LIB.he_plan_array(handle, which, None)
            out = np.zeros(count, dtype)
            _lib.LIB.he_plan_array(handle, which, ct.c_void_p(out.ctypes.data))
            return out
        scalars = get(30, np.int32)
        plan = {'ok': bool(scalars[0]), 'ne': int(scalars[1]), 'ntile': int(scalars[2]), 'ng': int(scalars[3]),
                'nlam': int(scalars[4]), 'maxm': int(scalars[5]), 'blkmax': int(scalars[6])}
        if plan['ok']:
            for which, name in enumerate(['estart', 'tstart', 'eoff', 'ereal', 'gch', 'wptr', 'wsrc', 'dwptr',
                                          'dwsrc', 'dwel', 'dwedge']):
                plan[name] = get(which, np.int32)
            plan['blocks'] = get(20, np.float64).view(np.complex128)
            plan['bblocks'] = get(21, np.float64).view(np.complex128)
            plan['wcoef'] = get(22, np.float64).reshape(-1, MIX_GROUP)
            plan['dwedge'] = plan['dwedge'].reshape(-1, MIX_GROUP)
            plan['gch'] = plan['gch'].reshape(-1, MIX_GROUP)
        return plan
    finally:
        _lib.LIB.he_plan_free(handle)


def emulate(h, x, field, velocity, P, beta=0, gamma=1):
    """numpy restatement of hpsi_radial_kernel + hpsi_mix_kernel on the plan P."""
    n, nc = h.n, h.nc
    es, ts, eoff = P['estart'], P['tstart'], P['eoff']
    ne, nt = P['ne'], P['ntile']
    assert es[0] == 0 and es[ne] == n and len(es) == ne + 1 and ts[0] == 0 and ts[nt] == ne
    psi = np.asarray(x).reshape((n, n, nc), order='F')
    size = lambda e: es[e + 1] - es[e] + 1 if e + 1 < ne else n - es[e]
    own = lambda e: (es[e + 1] if e + 1 < ne else n) - es[e]
    block = lambda arr, e: arr[eoff[e]:eoff[e] + size(e) ** 2].reshape(size(e), size(e))
    out = np.zeros_like(psi)
    W = [np.zeros_like(psi), np.zeros_like(psi)]
    f = np.asarray(field, float)
    a2 = float(f @ f)
    diag = np.asarray(h.diag).reshape((n, n, nc), order='F')
    for ti in range(nt):
        for tj in range(nt):
            ea, eb, fa, fb = ts[ti], ts[ti + 1], ts[tj], ts[tj + 1]
            r0, r1, c0, c1 = es[ea], es[eb], es[fa], es[fb]
            rs, cs, ro, co = min(r1 + 1, n) - r0, min(c1 + 1, n) - c0, r1 - r0, c1 - c0
            assert 0 < rs <= RAD_STRIDE and 0 < cs <= RAD_STRIDE and ro <= RAD_TMAX and co <= RAD_TMAX
            for ga, gb in ((ea, eb), (fa, fb)):   # staged element blocks of one axis fit the buffer
                staged = (size(ga - 1) if ga > 0 else 0) + sum(size(e) ** 2 for e in range(ga, gb))
                assert staged <= P['blkmax'] and gb - ga <= 4
            for c in range(nc):
                PS = psi[r0:r0 + rs, c0:c0 + cs, c]
                OS = np.zeros((ro, co), complex)
                WS = [np.zeros((ro, co), complex), np.zeros((ro, co), complex)]
                for axis, (ga, gb, base, other0, count) in enumerate([(ea, eb, r0, c0, co), (fa, fb, c0, r0, ro)]):
                    view = PS if axis == 0 else PS.T     # element index first
                    for e in range(ga, gb):
                        s, m, ow = es[e], size(e), own(e)
                        assert 0 <= s - base and s - base + m - 1 < view.shape[0]
                        T, B = block(P['blocks'], e), block(P['bblocks'], e)
                        for a0 in range(0, ow, RAD_CHUNK):
                            na = min(RAD_CHUNK, ow - a0)
                            xs = view[s - base:s - base + m, :count]
                            acc = T[a0:a0 + na] @ xs
                            accb = B[a0:a0 + na] @ xs
                            if a0 == 0 and e > 0:
                                sp, mp = es[e - 1], size(e - 1)
                                Tp, Bp = block(P['blocks'], e - 1)[mp - 1, :mp - 1], block(P['bblocks'], e - 1)[mp - 1, :mp - 1]
                                rows = np.arange(sp, sp + mp - 1)
                                left = np.array([view[r - base, :count] if r >= base else
                                                 (psi[r, other0:other0 + count, c] if axis == 0 else psi[other0:other0 + count, r, c])
                                                 for r in rows])
                                acc[0] += Tp @ left
                                accb[0] += Bp @ left
                            rows_out = slice(s - base + a0, s - base + a0 + na)
                            assert s - base + a0 + na <= (ro if axis == 0 else co)
                            if axis == 0:
                                OS[rows_out, :] = acc
                                WS[0][rows_out, :] = accb
                            else:
                                OS[:, rows_out] += acc.T
                                WS[1][:, rows_out] = accb.T
                x0 = PS[:ro, :co]
                v = OS + diag[r0:r1, c0:c1, c] * x0 + (a2 * x0 if velocity else 0)
                out[r0:r1, c0:c1, c] = v
                W[0][r0:r1, c0:c1, c], W[1][r0:r1, c0:c1, c] = WS
    # channel mixing (per point; the kernel's 128-point staging does not change the algebra)
    dcoef = np.asarray(h.dcoef).reshape(3, -1)
    coef = f @ dcoef if dcoef.shape[1] else np.zeros(0, complex)
    coef = np.where(np.abs(coef) < 1e-30, 0, coef)
    rad = np.asarray(h.rad).reshape((n, n, -1), order='F')
    r = np.asarray(h.r)
    ri, rj = r[:, None], r[None, :]
    final = np.zeros_like(psi)
    for g in range(P['ng']):
        chans = P['gch'][g]
        accs = [out[:, :, ch].copy() if ch >= 0 else None for ch in chans]
        for lam in range(P['nlam']):
            k0, k1 = P['wptr'][g * P['nlam'] + lam], P['wptr'][g * P['nlam'] + lam + 1]
            for d, ch in enumerate(chans):
                if ch < 0:
                    continue
                tsum = sum(P['wcoef'][k, d] * psi[:, :, P['wsrc'][k]] for k in range(k0, k1)) if k1 > k0 else 0
                accs[d] = accs[d] + rad[:, :, lam] * tsum
        for k in range(P['dwptr'][g], P['dwptr'][g + 1]):
            s, el = P['dwsrc'][k], P['dwel'][k]
            assert 0 <= s < nc and el in (1, 2)
            rr = ri if el == 1 else rj
            for d, ch in enumerate(chans):
                kk = P['dwedge'][k, d]
                if ch < 0 or kk < 0:
                    continue
                if not velocity:
                    accs[d] = accs[d] + coef[kk] * (rr * psi[:, :, s])
                else:
                    part = h.ldiff[kk] * (1 / (2 * rr)) * psi[:, :, s] + W[el - 1][:, :, s]
                    accs[d] = accs[d] + 1j * coef[kk] * part
        for d, ch in enumerate(chans):
            if ch >= 0:
                final[:, :, ch] = beta * psi[:, :, ch] + gamma * accs[d]
    covered = sorted(int(c) for c in P['gch'].ravel() if c >= 0)
    assert covered == list(range(nc))
    return final.ravel(order='F')


CASES = ['apply_ecs', 'apply_cut', 'apply_coupled']


@pytest.mark.parametrize('case', CASES)
@pytest.mark.parametrize('velocity', [False, True])
def test_tiled_plan_reproduces_the_oracle(case, velocity):
    g = golden(case)
    h = Tables(g)
    P = build_plan(h)
    assert P['ok']
    y = emulate(h, g['x'], g['field'], velocity, P)
    ref = cpu.tensor_apply(h, g['x'], g['field'], velocity)
    np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-11)


def test_tiled_plan_on_grid_with_tail_and_larger_elements():
    from laqphysics_b200.workloads import coupled, seeded_state
    h = coupled(np.linspace(0, 30, 16), 8, 3, 2, ecs_angle=.3, tail=12, cutoff_radii=(20., 25.))
    P = build_plan(h)
    assert P['ok'] and P['ne'] == 16 and P['maxm'] == 13
    x = seeded_state(h.size, 4)
    for velocity, field in ((False, (0, 0, .04)), (True, (0, 0, .3))):
        y = emulate(h, x, field, velocity, P, beta=.5 - .2j, gamma=.1j)
        ref = .5 * x - .2j * x + .1j * cpu.tensor_apply(h, x, field, velocity)
        np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-11)


def test_microbenchmark_plan_shape():
    from laqphysics_b200.workloads import hpsi_microbench
    h = hpsi_microbench()
    P = build_plan(h)
    assert P['ok'] and P['ne'] == 61 and P['maxm'] == 21
    # register blocking: 14 groups of <= 4 output channels (total-L block x l1-parity
    # classes) read 521 sources per point instead of 1071 edges
    assert P['ng'] == 14 and len(P['wsrc']) == 521
    est, ts = P['estart'], P['tstart']
    owned = [(est[ts[k + 1]] if ts[k + 1] < P['ne'] else h.n) - est[ts[k]] for k in range(P['ntile'])]
    assert max(owned) <= RAD_TMAX and sum(owned) == h.n


def test_plan_rejects_non_banded_kinetic_matrix():
    g = golden('apply_ecs')
    h = Tables(g)
    ptr, col, tv = h.ptr.copy(), h.col.copy(), h.tv.copy()
    # couple row 0 to the last node: no element structure any more
    col[ptr[1] - 1] = h.n - 1
    h.col = np.sort(col)
    assert not build_plan(h)['ok']
