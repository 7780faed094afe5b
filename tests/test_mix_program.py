"""The generated channel-mixing kernel, checked on the CPU.

The planner's mixing program (groups, blocks of multipoles, dipole edges; exported as
JSON) is run in numpy on top of the oracle's kinetic-plus-diagonal part and must
reproduce the oracle H·psi in both gauges; every edge of the tables must appear exactly
once.  The CUDA source generated from the program must compile with NVRTC for sm_100a
(no device needed).
"""
import ctypes as ct
import json

import numpy as np
import pytest

from conftest import Tables, golden
from oracle import cpu
from test_kinetic_plan import reference_kinetic


def planner(h):
    from laqphysics_b200 import _lib
    from laqphysics_b200.engine import _host_tables
    t = _host_tables(h)
    p = _lib.ptr
    return _lib, _lib.LIB.he_plan_build(h.n, h.nc, p(t['ptr']), p(t['col']), p(t['tv']), len(t['vc']), p(t['vptr']),
                                        p(t['vc']), p(t['vl']), p(t['vcoef']), t['nlam'], len(t['dc']),
                                        p(t['dptr']), p(t['dc']), p(t['de']), p(t['r']))


def mix_program(h):
    lib, handle = planner(h)
    try:
        n = lib.LIB.he_plan_mix_program(handle, None, 0)
        buf = ct.create_string_buffer(n + 1)
        lib.LIB.he_plan_mix_program(handle, buf, n + 1)
        return json.loads(buf.value.decode())
    finally:
        lib.LIB.he_plan_free(handle)


def mix_source(h, dipole_real=True):
    lib, handle = planner(h)
    try:
        n = lib.LIB.he_plan_mix_source(handle, int(dipole_real), None, 0)
        buf = ct.create_string_buffer(n + 1)
        lib.LIB.he_plan_mix_source(handle, int(dipole_real), buf, n + 1)
        return buf.value.decode()
    finally:
        lib.LIB.he_plan_free(handle)


def emulate_mix(h, x, field, velocity, prog, beta=0, gamma=1):
    """The generated kernel's arithmetic per group, vectorised over points."""
    n, nc = h.n, h.nc
    psi = np.asarray(x).reshape((n * n, nc), order='F')
    radial, W = reference_kinetic(h, x, velocity, a2=float(np.dot(field, field)))
    out = radial.reshape((n * n, nc), order='F').copy()
    W = [w.reshape((n * n, nc), order='F') for w in W]
    rad = np.asarray(h.rad).reshape((n * n, -1), order='F')
    dcoef = np.asarray(h.dcoef).reshape(3, -1, order='F') if len(h.dc) else np.zeros((3, 0))
    coef = np.asarray(field, float) @ dcoef if len(h.dc) else np.zeros(0)
    coef = np.where(np.abs(coef) < 1e-30, 0, coef)
    r = np.asarray(h.r)
    p = np.arange(n * n)
    rt = 1 / (2 * r) if velocity else r
    re = [rt[p % n], rt[p // n]]
    final = np.full((n * n, nc), np.nan, complex)
    seen_v, seen_d = [], []
    for G in prog:
        a = [out[:, c].copy() for c in G['out']]
        for B in G['blocks']:
            xs = [psi[:, s] for s in B['src']]
            for T in B['terms']:
                t = {}
                for d, s, w in zip(T['d'], T['s'], T['w']):
                    t[d] = t.get(d, 0) + w * xs[s]
                    seen_v.append((G['out'][d], B['src'][s], T['lam'], w))
                for d, v in t.items():
                    a[d] = a[d] + rad[:, T['lam']] * v
        for e, D in enumerate(G['dip']):
            u, z = {}, {}
            for d, s, k in zip(D['d'], D['s'], D['k']):
                seen_d.append(k)
                if velocity:
                    u[d] = u.get(d, 0) + 1j * coef[k] * h.ldiff[k] * psi[:, s]
                    z[d] = z.get(d, 0) + 1j * coef[k] * W[e][:, s]
                else:
                    u[d] = u.get(d, 0) + coef[k] * psi[:, s]
            for d in u:
                a[d] = a[d] + re[e] * u[d] + (z[d] if velocity else 0)
        for d, c in enumerate(G['out']):
            final[:, c] = beta * psi[:, c] + gamma * a[d]
    edges = sorted((c, int(h.vc[k]), int(h.vl[k]), float(np.real(h.vcoef[k])))
                   for c in range(nc) for k in range(h.vptr[c], h.vptr[c + 1]))
    assert sorted(seen_v) == edges, 'every Coulomb edge exactly once'
    assert sorted(seen_d) == list(range(len(h.dc))), 'every dipole edge exactly once'
    return final.ravel(order='F')


@pytest.mark.parametrize('case', ['apply_ecs', 'apply_cut', 'apply_coupled'])
@pytest.mark.parametrize('velocity', [False, True])
def test_mix_program_reproduces_the_oracle(case, velocity):
    g = golden(case)
    h = Tables(g)
    prog = mix_program(h)
    y = emulate_mix(h, g['x'], g['field'], velocity, prog)
    ref = cpu.tensor_apply(h, g['x'], g['field'], velocity)
    np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-11)


def test_mix_program_blocks_and_epilogue_on_larger_grid():
    from laqphysics_b200.workloads import coupled, seeded_state
    h = coupled(np.linspace(0, 30, 16), 8, 3, 2, ecs_angle=.3, tail=12, cutoff_radii=(20., 25.))
    prog = mix_program(h)
    assert max(len(B['src']) for G in prog for B in G['blocks']) <= 8
    assert max(len(G['out']) for G in prog) <= 8
    x = seeded_state(h.size, 5)
    for velocity, field in ((False, (0, 0, .04)), (True, (0, 0, .3))):
        y = emulate_mix(h, x, field, velocity, prog, beta=.5 - .2j, gamma=.1j)
        ref = (.5 - .2j) * x + .1j * cpu.tensor_apply(h, x, field, velocity)
        np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-11)


def test_microbenchmark_program_shape():
    from laqphysics_b200.workloads import hpsi_microbench
    h = hpsi_microbench()
    prog = mix_program(h)
    # the coupled basis splits into (total L, l1 parity) classes: even multipoles read the
    # class itself, odd ones its partner, so every block holds one class of sources
    assert sum(len(G['out']) for G in prog) == h.nc
    assert sum(len(T['d']) for G in prog for B in G['blocks'] for T in B['terms']) == len(h.vc)
    assert max(len(B['src']) for G in prog for B in G['blocks']) <= 8


@pytest.mark.parametrize('case', ['apply_coupled', 'microbench'])
def test_generated_source_compiles_for_sm100a(case):
    from laqphysics_b200 import _lib
    if case == 'microbench':
        from laqphysics_b200.workloads import hpsi_microbench
        h = hpsi_microbench()
    else:
        h = Tables(golden(case))
    for dipole_real in (True, False):
        src = mix_source(h, dipole_real)
        assert 'he_mix_d0' in src and 'he_mix_f1' in src
        log = ct.create_string_buffer(1 << 16)
        rc = _lib.LIB.he_nvrtc_check(src.encode(), log, len(log))
        assert rc == 0, log.value.decode()[:2000]
