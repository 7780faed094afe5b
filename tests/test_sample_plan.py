"""CPU model of the one-launch tSURFF sample's work decomposition (csrc/tsurff.cu,
surface_sample_kernel): tiles of 32 radial rows x 8 channels spread over the CTAs, the
frame rows each thread writes, the (label, outer) pairs each warp owns in the contraction,
the q entries each (CTA, thread) sums between the two waits, the Volkov items, and every
buffer index against its size — checked for the shapes the tests and the bench use and for
the limits (16 surface rows, 1024 contracted values)."""
import numpy as np
import pytest

TA, TC, THREADS, SC = 32, 8, 256, 8
NS_MAX, NQ_MAX = 16, 1024


def decomposition(n, nc, ns, nlab, nouter, ne, nang, grid):
    tiles_a, tiles = -(-n // TA), -(-n // TA) * -(-nc // TC)
    nq = nlab * nouter * ns
    frame = np.zeros((nc, ns, n), int)                    # writes per frame value
    q_partial = np.zeros((grid, nq), int)                 # contributions per CTA and q entry
    for b in range(grid):
        for tile in range(b, tiles, grid):
            a0, c0 = (tile % tiles_a) * TA, (tile // tiles_a) * TC
            for tid in range(THREADS):
                al, cl = tid % TA, tid // TA
                a, c = a0 + al, c0 + cl
                for s0 in range(0, ns, SC):
                    for u in range(SC):
                        s = s0 + u
                        if s >= ns:
                            continue
                        assert (s * TC + cl) * TA + al < ns * THREADS          # F in shared memory
                        if a < n and c < nc:
                            assert a + n * (s + ns * c) < n * ns * nc           # frame buffer
                            frame[c, s, a] += 1
            for warp in range(THREADS // 32):
                for jo in range(warp, nlab * nouter, THREADS // 32):
                    for s in range(ns):
                        assert jo * ns + s < nq <= NQ_MAX                       # Q in shared memory
                        q_partial[b, jo * ns + s] += 1
    with_tiles = min(grid, tiles)
    assert not q_partial[with_tiles:].any()                 # CTAs past the last tile hold nothing
    summed = np.zeros(nq, int)
    for b in range(grid):
        for tid in range(THREADS):
            for i in range(b + grid * tid, nq, grid * THREADS):
                summed[i] += 1
                for bb in range(with_tiles):
                    assert bb * nq + i < grid * nq                              # partial buffer
    items = np.zeros(nlab * ne * nang, int)
    for b in range(grid):
        for tid in range(THREADS):
            for idx in range(b * THREADS + tid, nlab * ne * nang, grid * THREADS):
                items[idx] += 1
    smem = (ns * THREADS + nq) * 16
    return frame, q_partial[:with_tiles].sum(axis=0), summed, items, smem, tiles


@pytest.mark.parametrize('n, nc, ns, nlab, nouter, ne, nang, grid', [
    (21, 6, 5, 3, 2, 7, 4, 1),            # golden Volkov case: one CTA
    (68, 11, 7, 3, 2, 240, 16, 45),       # the one-launch vs three-launch test
    (40, 4, 5, 3, 2, 21, 4, 2),           # tSURFF small case
    (560, 43, 10, 6, 6, 397, 32, 296),    # microbenchmark grid, 10 surface rows, He+ n <= 3
    (100, 17, 16, 4, 16, 5, 3, 9),        # the limits: 16 surface rows, nq = 1024
])
def test_every_output_once_and_every_index_in_bounds(n, nc, ns, nlab, nouter, ne, nang, grid):
    assert ns <= NS_MAX and nlab * nouter * ns <= NQ_MAX
    frame, per_q, summed, items, smem, tiles = decomposition(n, nc, ns, nlab, nouter, ne, nang, grid)
    assert np.all(frame == 1)
    assert np.all(per_q == tiles)          # every tile adds to every q entry once
    assert np.all(summed == 1)             # each q entry summed by exactly one thread
    assert np.all(items == 1)
    assert smem <= 227 * 1024
