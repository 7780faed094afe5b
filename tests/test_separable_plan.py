"""CPU model of the separable preconditioner's GEMM kernels (csrc/separable.cu), run before
any GPU use: the tile geometry and the epilogue's store indices (every output written once,
inside its channel and tile, never out of bounds), the TF32 split of the real embedding,
and the two-launch chain out_c = (M X_c)^T that composes A X B^T, against numpy in FP64.
"""
import numpy as np
import pytest

TG_BM, TG_BK, TG_BN_MAX = 128, 32, 256


def geometry(n, nc, sms=148):
    """he_separable_create's complex64 geometry: N tiles as few as the TMEM columns allow,
    more when the grid would leave SMs idle."""
    mtiles = -(-2 * n // TG_BM)
    ntn = -(-n // TG_BN_MAX)
    fill = -(-sms // (mtiles * nc))
    ntn = max(ntn, min(fill, max(1, n // 32)))
    bn = (-(-n // ntn) + 15) // 16 * 16
    ntn = -(-n // bn)
    ld = (2 * n + 3) // 4 * 4
    return ntn, bn, ld, -(-2 * n // TG_BK)


def tf32(x):
    """cvt.rna.tf32.f32 on float32 values (ties away from zero)."""
    b = np.asarray(x, np.float32).view(np.uint32)
    return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


@pytest.mark.parametrize('n, nc', [(7, 2), (132, 2), (132, 17), (150, 2), (257, 2), (300, 3), (560, 2), (560, 43)])
def test_epilogue_writes_every_output_once_in_bounds(n, nc):
    ntn, bn, ld, _ = geometry(n, nc)
    assert bn % 16 == 0 and 16 <= bn <= TG_BN_MAX and (ntn - 1) * bn < n <= ntn * bn
    assert ld % 4 == 0 and ld >= 2 * n
    hits = np.zeros((nc, n, n), int)
    mtiles = -(-2 * n // TG_BM)
    for c in range(nc):
        for mt in range(mtiles):
            for nt in range(ntn):
                j0 = nt * bn
                for thread in range(128):
                    row = mt * TG_BM + thread           # warp * 32 + lane
                    i, part = row >> 1, row & 1
                    for col in range(0, bn, 32):
                        assert col + 32 <= TG_BN_MAX     # TMEM columns allocated
                        jb = j0 + col + 16 * part
                        count = min(16, min(n, j0 + bn) - jb)
                        if i >= n or count <= 0:
                            continue
                        hits[c, i, jb:jb + count] += 1
                        # plane offsets of the stores stay inside row (c n + i)
                        assert 2 * (jb + count) <= ld
    assert np.all(hits == 1)


def embed(M):
    """Real embedding [[Re, -Im], [Im, Re]] interleaved: row 2i+p, column 2k+q."""
    n = M.shape[0]
    E = np.zeros((2 * n, 2 * n))
    E[0::2, 0::2], E[0::2, 1::2] = M.real, -M.imag
    E[1::2, 0::2], E[1::2, 1::2] = M.imag, M.real
    return E


def tf32_parts(x):
    hi = tf32(np.float32(x))
    return hi, tf32(np.float32(x) - hi)


def left_product_transposed(M, X, passes=3):
    """The kernel's out = (M X)^T for one channel through the real embedding, with the
    operand split and FP32 accumulation modelled in float64 (accumulation order aside)."""
    n = M.shape[0]
    Ah, Al = tf32_parts(embed(M))
    Xr = np.zeros((n, 2 * n), np.float32)               # row j = column j of X, (re, im) along k
    Xr[:, 0::2], Xr[:, 1::2] = X.T.real, X.T.imag
    Xh, Xl = tf32_parts(Xr)
    D = Ah.astype(float) @ Xh.T.astype(float)
    if passes == 3:
        D += Ah.astype(float) @ Xl.T.astype(float) + Al.astype(float) @ Xh.T.astype(float)
    C = D[0::2] + 1j * D[1::2]                           # (i, j)
    return C.T


@pytest.mark.parametrize('passes, bound', [(3, 2e-6), (1, 5e-3)])
def test_split_tf32_chain_matches_fp64(passes, bound):
    rng = np.random.default_rng(5)
    n = 40
    A, B = (rng.normal(size=(2, n, n)) + 1j * rng.normal(size=(2, n, n)))
    X = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    chain = left_product_transposed(B, left_product_transposed(A, X, passes), passes).T
    exact = A @ X @ B.T
    err = np.linalg.norm(chain.T - exact) / np.linalg.norm(exact)
    assert err < bound


def test_tf32_rounding_model():
    x = np.float32(1.0) + np.float32(2 ** -11)          # exactly half-way between TF32 neighbours
    assert tf32(x) == np.float32(1.0 + 2 ** -10)         # ties away from zero
    y = np.float32(np.pi)
    hi, lo = tf32_parts(y)
    assert abs(float(hi) + float(lo) - float(y)) < 2 ** -20 * abs(float(y))
