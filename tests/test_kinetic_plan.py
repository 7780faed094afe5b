"""The kinetic (TMA-staged) kernel's plan, checked on the CPU.

A numpy emulation follows hpsi_kinetic_kernel item by item: the staged box is cut from
psi exactly as the TMA copy would (start rounded down to 16 bytes, zero fill past the
grid), every shared-memory index the kernel forms is asserted to lie inside the box and
on a real node (never on zero fill), and the kinetic part, the diagonal and the
velocity-gauge stencils W1/W2 must reproduce the oracle-derived reference.
"""
import ctypes as ct

import numpy as np
import pytest

from conftest import Tables, golden

KIN_ROWS, KIN_SLOTS, KIN_NA, KIN_RELEMS = 64, 4, 10, 8


def kinetic_plan(h):
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
        s = get(31, np.int32)
        K = {'ok': bool(s[0]), 'ntr': int(s[1]), 'nct': int(s[2]), 'box_r64': int(s[3]), 'box_r32': int(s[4]),
             'box_c': int(s[5])}
        for which, name in ((0, 'estart'), (2, 'eoff'), (3, 'ereal'), (11, 'nodeelem'), (12, 'krow'),
                            (13, 'krbase'), (14, 'krcplx'), (15, 'kslot'), (16, 'kcbase'), (17, 'koff')):
            K[name] = get(which, np.int32)
        for which, name in ((23, 'tre'), (24, 'tim'), (25, 'bre'), (26, 'bim')):
            K[name] = get(which, np.float64)
        K['kslot'] = K['kslot'].reshape(-1, KIN_SLOTS, 3)
        return K
    finally:
        _lib.LIB.he_plan_free(handle)


def emulate_kinetic(h, x, K, velocity, a2=0.0, align=1):
    """Kinetic + diagonal (+ a2) and W1/W2 exactly as hpsi_kinetic_kernel forms them."""
    n, nc = h.n, h.nc
    ne = len(K['estart']) - 1
    es, eoff = K['estart'], K['eoff']
    msize = lambda e: (es[e + 1] + 1 if e + 1 < ne else n) - es[e]
    box_r = K['box_r64'] if align == 1 else K['box_r32']
    box_c = K['box_c']
    assert box_r <= 128 and box_c <= 256 and (align == 1 or box_r % 2 == 0)
    psi = np.asarray(x).reshape((n, n, nc), order='F')
    diag = np.asarray(h.diag).reshape((n, n, nc), order='F')
    out = np.full((n, n, nc), np.nan, complex)
    W = [np.full((n, n, nc), np.nan, complex), np.full((n, n, nc), np.nan, complex)]
    planes = {'T': (K['tre'], K['tim']), 'B': (K['bre'], K['bim'])}

    koff = K['koff']

    def coef(which, e, a, b, pair=False):   # X_e[a][b] from the padded transposed planes
        re, im = planes[which]
        m = msize(e)
        k = koff[e] + b * (m + (m & 1)) + a
        assert 0 <= a < m and 0 <= b < m and k < koff[e + 1]
        if pair:                             # the kernel loads (k, k+1) as one vector
            assert k % 2 == 0 and k + 1 < len(re)
        return re[k] + 1j * im[k]

    covered = np.zeros((n, n), int)
    for tr in range(K['ntr']):
        ea, eb = K['krow'][tr], K['krow'][tr + 1]
        r0, r1 = es[ea], (es[eb] if eb < ne else n)
        x0 = K['krbase'][tr] // align * align
        assert (x0 * 16 // align) % 16 == 0 and x0 >= 0
        assert eb - ea <= KIN_RELEMS
        for tc in range(K['nct']):
            y0 = K['kcbase'][tc]
            valid = np.zeros((box_c, box_r), bool)   # S[col][row] holds a real node
            for cc in range(box_c):
                for rr in range(box_r):
                    valid[cc, rr] = x0 + rr < n and y0 + cc < n

            def S(c, col, row):
                cc, rr = col - y0, row - x0
                assert 0 <= cc < box_c and 0 <= rr < box_r and valid[cc, rr], (col, row, y0, x0)
                return psi[row, col, c]

            c0 = es[K['kslot'][tc, 0, 0]] + K['kslot'][tc, 0, 1]
            assert K['kslot'][tc, :, 2].sum() <= KIN_SLOTS * KIN_NA
            for slot in range(KIN_SLOTS):
                f, a0, na = K['kslot'][tc, slot]
                if na == 0:
                    continue
                assert na <= KIN_NA
                sf, mf = es[f], msize(f)
                cq0 = sf + a0
                for lane in range(KIN_ROWS):
                    i = r0 + lane
                    if i >= r1:
                        continue
                    covered[i, cq0:cq0 + na] += 1
                    for c in range(nc):
                        def r2(which):
                            acc = np.zeros(na, complex)
                            assert a0 % 2 == 0
                            for b in range(mf):
                                xv = S(c, sf + b, i)
                                for q in range(na):
                                    acc[q] += coef(which, f, a0 + q, b, pair=q % 2 == 0) * xv
                            if a0 == 0 and f > 0:
                                fp = f - 1
                                sp, mp = es[fp], sf - es[fp] + 1
                                for b in range(mp - 1):
                                    acc[0] += coef(which, fp, mp - 1, b) * S(c, sp + b, i)
                            return acc

                        def r1_(which):
                            acc = np.zeros(na, complex)
                            e = K['nodeelem'][i]
                            se, me = es[e], msize(e)
                            ai = i - se
                            assert 0 <= ai < me
                            for b in range(me):
                                t = coef(which, e, ai, b)
                                for q in range(na):
                                    acc[q] += t * S(c, cq0 + q, se + b)
                            if ai == 0 and e > 0:   # kernel: bridge partials (kinetic) or in-lane (W1)
                                assert 0 <= e - max(ea, 1) < KIN_RELEMS and 0 <= cq0 - c0 and cq0 - c0 + na <= KIN_SLOTS * KIN_NA
                                ep = e - 1
                                sp, mp = es[ep], se - es[ep] + 1
                                for b in range(mp - 1):
                                    t = coef(which, ep, mp - 1, b)
                                    for q in range(na):
                                        acc[q] += t * S(c, cq0 + q, sp + b)
                            return acc

                        if velocity:
                            W[1][i, cq0:cq0 + na, c] = r2('B')
                            W[0][i, cq0:cq0 + na, c] = r1_('B')
                        acc = r2('T') + r1_('T')
                        for q in range(na):
                            j = cq0 + q
                            xv = S(c, j, i)
                            v = acc[q] + diag[i, j, c] * xv
                            if velocity:
                                v += a2 * xv
                            out[i, j, c] = v
    assert (covered == 1).all(), 'every output point is owned by exactly one (tile, slot, lane)'
    return out, W


def reference_kinetic(h, x, velocity, a2=0.0):
    """Kinetic + diagonal (+ |A|^2) and the commutator stencils from the CSR tables."""
    import scipy.sparse as sp
    n, nc = h.n, h.nc
    T = sp.csr_matrix((np.asarray(h.tv), np.asarray(h.col), np.asarray(h.ptr)), shape=(n, n)).toarray()
    r = np.asarray(h.r)
    B = T * (r[None, :] - r[:, None])
    psi = np.asarray(x).reshape((n, n, nc), order='F')
    diag = np.asarray(h.diag).reshape((n, n, nc), order='F')
    out = np.einsum('ab,bjc->ajc', T, psi) + np.einsum('ab,ibc->iac', T, psi) + diag * psi
    if velocity:
        out = out + a2 * psi
    W1 = np.einsum('ab,bjc->ajc', B, psi)
    W2 = np.einsum('ab,ibc->iac', B, psi)
    return out, (W1, W2)


@pytest.mark.parametrize('case', ['apply_ecs', 'apply_cut', 'apply_coupled'])
@pytest.mark.parametrize('align', [1, 2])
def test_kinetic_plan_reproduces_the_stencils(case, align):
    g = golden(case)
    h = Tables(g)
    K = kinetic_plan(h)
    assert K['ok']
    x = np.asarray(g['x'])
    out, W = emulate_kinetic(h, x, K, True, a2=0.3, align=align)
    ref, Wref = reference_kinetic(h, x, True, a2=0.3)
    np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-11)
    np.testing.assert_allclose(W[0], Wref[0], rtol=1e-12, atol=1e-11)
    np.testing.assert_allclose(W[1], Wref[1], rtol=1e-12, atol=1e-11)


def test_kinetic_plan_with_tail_and_split_slots():
    from laqphysics_b200.workloads import coupled, seeded_state
    # a 24-point exterior tail element: its 25 owned columns split into three slots, the
    # last of which starts a column tile in the middle of the element
    h = coupled(np.linspace(0, 24, 7), 6, 1, 1, ecs_angle=.3, tail=24, cutoff_radii=(12., 15.))
    K = kinetic_plan(h)
    assert K['ok'] and K['kslot'][-1, 0, 1] > 0
    x = seeded_state(h.size, 7)
    for align in (1, 2):
        out, W = emulate_kinetic(h, x, K, True, a2=0.05, align=align)
        ref, Wref = reference_kinetic(h, x, True, a2=0.05)
        np.testing.assert_allclose(out, ref, rtol=1e-12, atol=1e-11)
        np.testing.assert_allclose(W[0], Wref[0], rtol=1e-12, atol=1e-11)
        np.testing.assert_allclose(W[1], Wref[1], rtol=1e-12, atol=1e-11)


def test_microbenchmark_kinetic_tiles():
    from laqphysics_b200.workloads import hpsi_microbench
    h = hpsi_microbench()
    K = kinetic_plan(h)
    assert K['ok']
    est, krow = K['estart'], K['krow']
    ne = len(est) - 1
    owned = [(est[krow[t + 1]] if krow[t + 1] < ne else h.n) - est[krow[t]] for t in range(K['ntr'])]
    assert max(owned) <= KIN_ROWS and sum(owned) == h.n
    assert K['kslot'][:, :, 2].sum() == h.n
    # two staged boxes per CTA and two CTAs per SM fit the 228 KB of an SM
    stage = -(-K['box_r64'] * K['box_c'] * 16 // 128) * 128
    bridge = KIN_RELEMS * KIN_SLOTS * KIN_NA * 16
    assert 2 * (2 * stage + bridge + 16 + 128 + 1024) <= 228 * 1024, (K['box_r64'], K['box_c'])


# --------------------------------------------------------------------------------------
# Banded FP64 tensor-core kernel (hpsi_band_kernel)
# --------------------------------------------------------------------------------------
BAND_G, BAND_KS, BAND_TR, BAND_TC = 8, 8, 64, 32


def band_plan(h):
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
        s = get(34, np.int32)
        B = dict(zip(('ok', 'ngroup', 'ntr', 'nct', 'box_r', 'box_r32', 'box_c'), (int(v) for v in s)))
        for which, name in ((18, 'glo'), (19, 'gks'), (29, 'greal'), (32, 'brbase'), (33, 'bcbase')):
            B[name] = get(which, np.int32)
        for which, name in ((27, 'frag'), (28, 'fragb')):
            B[name] = get(which, np.float64).view(np.complex128).reshape(-1, BAND_KS, 32)
        return B
    finally:
        _lib.LIB.he_plan_free(handle)


def emulate_band(h, x, B, velocity, a2=0.0, channels=None, align=1):
    """hpsi_band_kernel item by item: mma fragments formed lane by lane from the staged box
    (every index asserted inside it), C[j][i] accumulated as 8x4 @ 4x8 products.  align=2
    is the complex64 form (box rows start on an even node, pitch box_r32)."""
    n, nc = h.n, h.nc
    G, P, BC = B['ngroup'], (B['box_r'] if align == 1 else B['box_r32']), B['box_c']
    assert align == 1 or (P % 2 == 0 and n % 2 == 0)
    assert P % 8 == 4 and 2 * P <= 256 and BC <= 256
    psi = np.asarray(x).reshape((n, n, nc), order='F')
    diag = np.asarray(h.diag).reshape((n, n, nc), order='F')
    chans = range(nc) if channels is None else channels
    out = {c: np.full((n, n), np.nan, complex) for c in chans}
    W = [{c: np.full((n, n), np.nan, complex) for c in chans} for _ in range(2)]
    lanes = np.arange(32)
    lr, lk = lanes >> 2, lanes & 3
    for tr in range(B['ntr']):
        x0 = B['brbase'][tr] // align * align
        for tc in range(B['nct']):
            y0 = B['bcbase'][tc]
            for c in chans:
                box = np.zeros((P, BC), complex)        # box[row - x0, col - y0], zero fill past the grid
                rr, cc = np.arange(P) + x0, np.arange(BC) + y0
                box[np.ix_(rr < n, cc < n)] = psi[np.ix_(rr[rr < n], cc[cc < n], [c])][:, :, 0]

                def S(rows, cols):
                    rows, cols = np.asarray(rows), np.asarray(cols)
                    assert (rows >= x0).all() and (rows < x0 + P).all() and (cols >= y0).all() and (cols < y0 + BC).all()
                    return box[rows - x0, cols - y0]

                for w in range(BAND_TR // BAND_G):
                    gr = tr * (BAND_TR // BAND_G) + w
                    if gr >= G:
                        continue
                    i0 = gr * BAND_G
                    for q in range(BAND_TC // BAND_G):
                        gc = tc * (BAND_TC // BAND_G) + q
                        if gc >= G:
                            break
                        j0 = gc * BAND_G

                        def r1(frag):
                            C = np.zeros((8, 8), complex)
                            for s in range(B['gks'][gr]):
                                a = np.zeros((8, 4), complex)
                                b = np.zeros((4, 8), complex)
                                a[lr, lk] = S(B['glo'][gr] + 4 * s + lk, j0 + lr)   # A[m][k] = S[r][j0+m]
                                b[lk, lr] = frag[gr, s, lanes]                        # B[k][n] = T[i0+n][r]
                                C += a @ b
                            return C

                        def r2(frag):
                            C = np.zeros((8, 8), complex)
                            for s in range(B['gks'][gc]):
                                a = np.zeros((8, 4), complex)
                                b = np.zeros((4, 8), complex)
                                a[lr, lk] = frag[gc, s, lanes]                        # A[m][k] = T[j0+m][r']
                                b[lk, lr] = S(i0 + lr, B['glo'][gc] + 4 * s + lk)    # B[k][n] = S[i0+n][r']
                                C += a @ b
                            return C

                        def put(dst, C):
                            for m in range(8):
                                for nn_ in range(8):
                                    i, j = i0 + nn_, j0 + m
                                    if i < n and j < n:
                                        dst[i, j] = C[m, nn_]

                        if velocity:
                            put(W[0][c], r1(B['fragb']))
                            put(W[1][c], r2(B['fragb']))
                        C = r1(B['frag']) + r2(B['frag'])
                        for m in range(8):
                            for nn_ in range(8):
                                i, j = i0 + nn_, j0 + m
                                if i < n and j < n:
                                    xv = S(i, j)
                                    out[c][i, j] = C[m, nn_] + diag[i, j, c] * xv + (a2 * xv if velocity else 0)
    return out, W


@pytest.mark.parametrize('case', ['apply_ecs', 'apply_cut', 'apply_coupled'])
@pytest.mark.parametrize('align', [1, 2])
def test_band_plan_reproduces_the_stencils(case, align):
    g = golden(case)
    h = Tables(g)
    B = band_plan(h)
    assert B['ok']
    if align == 2 and h.n % 2:
        pytest.skip('complex64 TMA rows need an even node count')
    x = np.asarray(g['x'])
    chans = sorted({0, h.nc - 1})
    out, W = emulate_band(h, x, B, True, a2=0.3, channels=chans, align=align)
    ref, Wref = reference_kinetic(h, x, True, a2=0.3)
    for c in chans:
        np.testing.assert_allclose(out[c], ref[:, :, c], rtol=1e-12, atol=1e-11)
        np.testing.assert_allclose(W[0][c], Wref[0][:, :, c], rtol=1e-12, atol=1e-11)
        np.testing.assert_allclose(W[1][c], Wref[1][:, :, c], rtol=1e-12, atol=1e-11)


def test_band_plan_with_tail_and_ragged_group():
    from laqphysics_b200.workloads import coupled, seeded_state
    # n = 6*6 + 24 + 1 - 1 is not a multiple of 8: the last row group is ragged
    h = coupled(np.linspace(0, 24, 7), 6, 1, 1, ecs_angle=.3, tail=24, cutoff_radii=(12., 15.))
    B = band_plan(h)
    assert B['ok'] and h.n % 8 != 0
    x = seeded_state(h.size, 9)
    ref, Wref = reference_kinetic(h, x, True, a2=0.05)
    for align in (1, 2) if h.n % 2 == 0 else (1,):
        out, W = emulate_band(h, x, B, True, a2=0.05, channels=[0, h.nc - 1], align=align)
        for c in (0, h.nc - 1):
            np.testing.assert_allclose(out[c], ref[:, :, c], rtol=1e-12, atol=1e-11)
            np.testing.assert_allclose(W[0][c], Wref[0][:, :, c], rtol=1e-12, atol=1e-11)
            np.testing.assert_allclose(W[1][c], Wref[1][:, :, c], rtol=1e-12, atol=1e-11)


def test_microbenchmark_band_tiles():
    from laqphysics_b200.workloads import hpsi_microbench
    h = hpsi_microbench()
    B = band_plan(h)
    assert B['ok'] and B['ngroup'] == 70 and B['ntr'] == 9 and B['nct'] == 18
    assert B['gks'].max() <= BAND_KS
    stage = -(-B['box_r'] * B['box_c'] * 16 // 128) * 128
    smem = 2 * stage + 4 * BAND_KS * 32 * 16 + 16 + 128
    assert smem + 1024 <= 228 * 1024, (B['box_r'], B['box_c'], smem)
