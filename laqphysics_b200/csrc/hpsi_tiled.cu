// Tiled two-electron H·psi for sm_100a (the production path; hamiltonian.cu keeps the
// generic one-thread-per-output kernel for tables the planner cannot express).
//
// H psi is split by the structure of the operator (python/torch_backend.py:109-131,
// src/kernels.f90:132-171):
//
//   hpsi_radial_kernel  per channel, element-aligned 2D tiles staged in shared memory:
//                       kinetic energy of electron 1 and 2 (the FE-DVR matrix is block
//                       banded: a row couples only to nodes of its element, a bridge row
//                       to two elements), the separable or tabulated diagonal and |A|^2;
//                       in the velocity gauge also W_e = B_e psi with B = T (r_b - r_a),
//                       the [T, r] commutator stencils of src/kernels.f90:153-168.
//                       A warp works on one element and 32 lines; each lane keeps the
//                       element's inputs and all its output rows in registers.
//   hpsi_mix_kernel     per point, all channels of MIX_NP points staged in shared memory:
//                       Coulomb multipoles sum_lam rad_lam sum_c' V_lam[c,c'] psi_c' and the
//                       dipole couplings, register-blocked over MIX_GROUP output channels
//                       that share source channels ("wide edges") and two points per lane,
//                       then the epilogue out = beta psi + gamma (H psi).
//
// psi is read once from DRAM by each kernel; the radial result travels through `out`.
// Every table an inner loop touches (element blocks, wide edges, dipole coefficients)
// is staged in shared memory first, so the loops issue no global loads.
#include <algorithm>

#include "common.cuh"
#include "hpsi_tiled.cuh"
#include "operator.cuh"

namespace he {

constexpr int RAD_THREADS = 256;
constexpr int RAD_STRIDE = RAD_TMAX + 1;   // odd row stride (complex elements): conflict-free column reads
constexpr int EMAX = 12;                   // elements up to EMAX nodes run the fully unrolled register path
constexpr int MIX_NP = 64;                 // points per mixing CTA (two per lane)
constexpr int MIX_THREADS = 128;

// Per-axis description of a radial tile, built in shared memory by the CTA.
struct AxisTile {
    int ga, gb, count;                   // element range, gb - ga
    int lines, linechunks;               // lines of the other axis, ceil(lines / 32)
    int s[RAD_ELEMS], m[RAD_ELEMS], own[RAD_ELEMS], real[RAD_ELEMS], chunks[RAD_ELEMS];
    int off[RAD_ELEMS];                  // offset of the element's block in the staged blocks
    int tasks[RAD_ELEMS + 1];            // prefix sums of per-lane items (row chunks x lines)
    int prev, prev_m, prev_real, prev_off;   // previous element (bridge row), -1 if none
};

template <typename R>
__device__ void stage_axis(const TiledPlan<R> &pl, AxisTile &ax, int ga, int gb, int lines, cplx<R> *dst,
                           cplx<R> *dstB, bool vel)
{
    const int n = pl.n, ne = pl.ne;
    if (threadIdx.x == 0) {
        ax.ga = ga; ax.gb = gb; ax.count = gb - ga;
        ax.lines = lines; ax.linechunks = (lines + 31) / 32;
        int off = 0;
        ax.prev = ga > 0 ? ga - 1 : -1;
        ax.prev_off = 0; ax.prev_m = 0; ax.prev_real = 1;
        if (ga > 0) {
            const int e = ga - 1;
            ax.prev_m = e + 1 < ne ? pl.estart[e + 1] - pl.estart[e] + 1 : n - pl.estart[e];
            ax.prev_real = pl.ereal[e];
            ax.prev_off = 0;
            off = ax.prev_m;
        }
        ax.tasks[0] = 0;
        for (int k = 0; k < ax.count; ++k) {
            const int e = ga + k;
            ax.s[k] = pl.estart[e];
            ax.m[k] = e + 1 < ne ? pl.estart[e + 1] - pl.estart[e] + 1 : n - pl.estart[e];
            ax.own[k] = (e + 1 < ne ? pl.estart[e + 1] : n) - pl.estart[e];
            ax.real[k] = pl.ereal[e];
            ax.chunks[k] = ax.m[k] <= EMAX ? 1 : (ax.own[k] + EMAX - 1) / EMAX;
            ax.off[k] = off;
            off += ax.m[k] * ax.m[k];
            ax.tasks[k + 1] = ax.tasks[k] + ax.chunks[k] * ax.lines;   // per-lane items
        }
    }
    __syncthreads();
    if (ax.prev >= 0) {
        const int mp = ax.prev_m;
        const size_t src = (size_t)pl.eoff[ax.prev] + (size_t)(mp - 1) * mp;
        for (int b = threadIdx.x; b < mp; b += blockDim.x) {
            dst[b] = pl.blocks[src + b];
            if (vel) dstB[b] = pl.bblocks[src + b];
        }
    }
    for (int k = 0; k < ax.count; ++k) {
        const int mm = ax.m[k] * ax.m[k];
        const size_t src = pl.eoff[ax.ga + k];
        for (int q = threadIdx.x; q < mm; q += blockDim.x) {
            dst[ax.off[k] + q] = pl.blocks[src + q];
            if (vel) dstB[ax.off[k] + q] = pl.bblocks[src + q];
        }
    }
}

// ---------------------------------------------------------------------------------
// Asynchronous global -> shared copies (cp.async, zero fill when src_bytes == 0).
// ---------------------------------------------------------------------------------
template <int BYTES> __device__ __forceinline__ void cp_async(void *smem, const void *gmem, int src_bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// acc[a] = sum_b blk[a M + b] x[b], a < na, for an element of exactly M nodes.
template <typename R, bool REAL, int M>
__device__ __forceinline__ void rows_fixed(const cplx<R> *blk, int na, const cplx<R> *xs, int xstride,
                                           cplx<R> (&acc)[EMAX])
{
    cplx<R> x[M];
#pragma unroll
    for (int b = 0; b < M; ++b) x[b] = xs[b * xstride];
#pragma unroll
    for (int a = 0; a < M; ++a) {
        if (a < na) {
            const cplx<R> *row = blk + a * M;
            cplx<R> s = mk<R>(0, 0);
#pragma unroll
            for (int b = 0; b < M; ++b) s = REAL ? rfma<R>(row[b].x, x[b], s) : cfma<R>(row[b], x[b], s);
            acc[a] = s;
        }
    }
}

// Same for any m <= EMAX (predicated; used for element sizes without a fixed variant).
template <typename R, bool REAL>
__device__ __forceinline__ void rows_any(const cplx<R> *blk, int m, int na, const cplx<R> *xs, int xstride,
                                         cplx<R> (&acc)[EMAX])
{
    cplx<R> x[EMAX];
#pragma unroll
    for (int b = 0; b < EMAX; ++b) x[b] = b < m ? xs[b * xstride] : mk<R>(0, 0);
#pragma unroll
    for (int a = 0; a < EMAX; ++a) {
        if (a < na) {
            const cplx<R> *row = blk + a * m;
            cplx<R> s = mk<R>(0, 0);
#pragma unroll
            for (int b = 0; b < EMAX; ++b)
                if (b < m) s = REAL ? rfma<R>(row[b].x, x[b], s) : cfma<R>(row[b], x[b], s);
            acc[a] = s;
        }
    }
}

template <typename R, bool REAL>
__device__ __forceinline__ void rows_small(const cplx<R> *blk, int m, int na, const cplx<R> *xs, int xstride,
                                           cplx<R> (&acc)[EMAX])
{
    switch (m) {   // m is warp uniform: the common FE orders get exact unrolls
    case 8: rows_fixed<R, REAL, 8>(blk, na, xs, xstride, acc); break;
    case 9: rows_fixed<R, REAL, 9>(blk, na, xs, xstride, acc); break;
    case 10: rows_fixed<R, REAL, 10>(blk, na, xs, xstride, acc); break;
    case 11: rows_fixed<R, REAL, 11>(blk, na, xs, xstride, acc); break;
    default: rows_any<R, REAL>(blk, m, na, xs, xstride, acc); break;
    }
}

// Rows [a0, a0 + na) of element k applied to one line, with the previous element's part
// of the bridge row added when a0 == 0.  `blocks` is the staged T (or B) block set,
// `prevrow` the previous element's last row of the same kind.
template <typename R, bool ROWS>
__device__ __forceinline__ void element_line(const AxisTile &ax, int k, const cplx<R> *blocks, const cplx<R> *prevrow,
                                             const cplx<R> *PS, int base, int r0, int c0, int n, const cplx<R> *pc,
                                             int line, int a0, int na, cplx<R> (&acc)[EMAX])
{
    const int s = ax.s[k], m = ax.m[k];
    const cplx<R> *blk = blocks + ax.off[k];
    const cplx<R> *xs = ROWS ? PS + (s - base) * RAD_STRIDE + line : PS + line * RAD_STRIDE + (s - base);
    const int xstride = ROWS ? RAD_STRIDE : 1;
#pragma unroll
    for (int q = 0; q < EMAX; ++q) acc[q] = mk<R>(0, 0);
    if (m <= EMAX) {
        if (ax.real[k]) rows_small<R, true>(blk, m, na, xs, xstride, acc);
        else rows_small<R, false>(blk, m, na, xs, xstride, acc);
    } else {   // large element (the exterior-scaled tail): stream over its nodes
        const bool real = ax.real[k];
        for (int b = 0; b < m; ++b) {
            const cplx<R> x = xs[b * xstride];
#pragma unroll
            for (int q = 0; q < EMAX; ++q) {
                if (q < na) {
                    const cplx<R> tv = blk[(a0 + q) * m + b];
                    acc[q] = real ? rfma<R>(tv.x, x, acc[q]) : cfma<R>(tv, x, acc[q]);
                }
            }
        }
    }
    if (a0 == 0 && (k > 0 || ax.prev >= 0)) {   // bridge row s: the previous element's part
        const cplx<R> *bp;
        int mp, sp;
        bool rp;
        if (k > 0) {
            mp = ax.m[k - 1]; sp = ax.s[k - 1]; rp = ax.real[k - 1];
            bp = blocks + ax.off[k - 1] + (mp - 1) * mp;
        } else {
            mp = ax.prev_m; sp = s - (mp - 1); rp = ax.prev_real;
            bp = prevrow;
        }
        for (int b = 0; b < mp - 1; ++b) {
            const int node = sp + b;   // global index along this axis
            cplx<R> x;
            if (node >= base) x = ROWS ? PS[(node - base) * RAD_STRIDE + line] : PS[line * RAD_STRIDE + node - base];
            else x = ROWS ? pc[(size_t)node + (size_t)n * (c0 + line)] : pc[(size_t)(r0 + line) + (size_t)n * node];
            acc[0] = rp ? rfma<R>(bp[b].x, x, acc[0]) : cfma<R>(bp[b], x, acc[0]);
        }
    }
}

// One direction of the radial stencil on the staged tile.  ROWS = electron 1 (lines are
// owned columns, the element index runs along rows), else electron 2.  The kinetic
// result goes to OS; in the velocity gauge a second pass applies B and writes W.
template <typename R, bool VEL, bool ROWS>
__device__ void radial_phase(const AxisTile &ax, const cplx<R> *BLK, const cplx<R> *BLKB, const cplx<R> *PS,
                             cplx<R> *OS, int base, int r0, int c0, int n, const cplx<R> *pc, cplx<R> *wout,
                             size_t nn, int c)
{
    // Items are (element k, row chunk, line), line fastest, flattened over the tile so that
    // every lane of every warp has one; neighbouring lanes share the element's block.
    const int nitems = ax.tasks[ax.count];
    for (int item = threadIdx.x; item < nitems; item += blockDim.x) {
        int k = 0;
        while (k + 1 < ax.count && item >= ax.tasks[k + 1]) ++k;
        const int rest = item - ax.tasks[k];
        const int line = rest % ax.lines, chunk = rest / ax.lines;
        const int s = ax.s[k];
        const int a0 = chunk * EMAX, na = min(EMAX, ax.own[k] - a0);
        cplx<R> acc[EMAX];
        element_line<R, ROWS>(ax, k, BLK, BLK + ax.prev_off, PS, base, r0, c0, n, pc, line, a0, na, acc);
#pragma unroll
        for (int q = 0; q < EMAX; ++q) {
            if (q < na) {
                const int node = s - base + a0 + q;
                const int row = ROWS ? node : line, col = ROWS ? line : node;
                if (ROWS) OS[row * RAD_STRIDE + col] = acc[q];
                else OS[row * RAD_STRIDE + col] = cadd<R>(OS[row * RAD_STRIDE + col], acc[q]);
            }
        }
        if (VEL) {
            element_line<R, ROWS>(ax, k, BLKB, BLKB + ax.prev_off, PS, base, r0, c0, n, pc, line, a0, na, acc);
#pragma unroll
            for (int q = 0; q < EMAX; ++q) {
                if (q < na) {
                    const int node = s - base + a0 + q;
                    const int row = ROWS ? node : line, col = ROWS ? line : node;
                    wout[(size_t)(r0 + row) + (size_t)n * (c0 + col) + nn * c] = acc[q];
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------
// Radial stencil kernel.  grid = (ntile * ntile, ceil(nc / RAD_CH)); a CTA owns one tile
// and RAD_CH channels.  The staged psi of channel c+1 streams in (cp.async, second
// buffer) while channel c is computed.
// ---------------------------------------------------------------------------------
constexpr int RAD_CH = 4;

template <typename R>
__device__ __forceinline__ void radial_prefetch(const cplx<R> *pc, cplx<R> *dst, int r0, int c0, int rs, int cs, int n)
{
    for (int idx = threadIdx.x; idx < rs * cs; idx += blockDim.x) {
        const int a = idx % rs, b = idx / rs;
        cp_async<sizeof(cplx<R>)>(dst + a * RAD_STRIDE + b, pc + (size_t)(r0 + a) + (size_t)n * (c0 + b),
                                  (int)sizeof(cplx<R>));
    }
    cp_async_commit();
}

template <typename R, bool VEL, bool SEP>
__global__ void __launch_bounds__(RAD_THREADS, 2)
hpsi_radial_kernel(const DeviceTables<R> t, const TiledPlan<R> pl, const cplx<R> *__restrict__ psi,
                   cplx<R> *__restrict__ out, cplx<R> *__restrict__ w1, cplx<R> *__restrict__ w2, R a2, int blkmax)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R> *PSB = reinterpret_cast<cplx<R> *>(smem_raw);          // two staged psi buffers
    cplx<R> *OS = PSB + 2 * RAD_STRIDE * RAD_STRIDE;
    cplx<R> *B0 = OS + RAD_TMAX * RAD_STRIDE;        // electron-1 blocks (T), then B if VEL
    cplx<R> *B0B = B0 + blkmax;
    cplx<R> *B1 = B0 + (VEL ? 2 : 1) * blkmax;       // electron-2 blocks
    cplx<R> *B1B = B1 + blkmax;
    __shared__ AxisTile ax0, ax1;

    const int n = pl.n;
    const int ti = blockIdx.x % pl.ntile, tj = blockIdx.x / pl.ntile;
    const int cbeg = blockIdx.y * RAD_CH, cend = min(pl.nc, cbeg + RAD_CH);
    const int ea = pl.tstart[ti], eb = pl.tstart[ti + 1];
    const int fa = pl.tstart[tj], fb = pl.tstart[tj + 1];
    const int r0 = pl.estart[ea], r1 = pl.estart[eb];          // owned rows [r0, r1)
    const int c0 = pl.estart[fa], c1 = pl.estart[fb];          // owned cols [c0, c1)
    const int rs = min(r1 + 1, n) - r0, cs = min(c1 + 1, n) - c0;   // staged extents (+ right bridge)
    const int ro = r1 - r0, co = c1 - c0;
    const size_t nn = (size_t)n * n;

    radial_prefetch<R>(psi + nn * cbeg, PSB, r0, c0, rs, cs, n);
    stage_axis<R>(pl, ax0, ea, eb, co, B0, B0B, VEL);
    stage_axis<R>(pl, ax1, fa, fb, ro, B1, B1B, VEL);
    for (int c = cbeg; c < cend; ++c) {
        const int buf = (c - cbeg) & 1;
        cplx<R> *PS = PSB + buf * RAD_STRIDE * RAD_STRIDE;
        if (c + 1 < cend) {
            radial_prefetch<R>(psi + nn * (c + 1), PSB + (buf ^ 1) * RAD_STRIDE * RAD_STRIDE, r0, c0, rs, cs, n);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const cplx<R> *pc = psi + nn * c;
        radial_phase<R, VEL, true>(ax0, B0, B0B, PS, OS, r0, r0, c0, n, pc, w1, nn, c);
        __syncthreads();
        radial_phase<R, VEL, false>(ax1, B1, B1B, PS, OS, c0, r0, c0, n, pc, w2, nn, c);
        __syncthreads();
        for (int idx = threadIdx.x; idx < ro * co; idx += blockDim.x) {
            const int a = idx % ro, b = idx / ro;
            const int i = r0 + a, j = c0 + b;
            const size_t p = (size_t)i + (size_t)n * j;
            const cplx<R> x = PS[a * RAD_STRIDE + b];
            const cplx<R> d = SEP ? cadd<R>(ldg<R>(t.d1 + i + (size_t)n * c), ldg<R>(t.d2 + j + (size_t)n * c))
                                  : ldg<R>(t.diag + p + nn * c);
            cplx<R> v = cfma<R>(d, x, OS[a * RAD_STRIDE + b]);
            if (VEL) v = rfma<R>(a2, x, v);
            out[p + nn * c] = v;
        }
        __syncthreads();   // PS[buf] and OS are reused by the next channels
    }
}

// ---------------------------------------------------------------------------------
// Channel-mixing kernel.  Persistent over tiles of MIX_NP consecutive flattened points
// p = i + n j; one warp per output group; the group tables are staged once per CTA and
// the psi/rad tile of the next point block streams in (cp.async) while the current one
// is computed.
// Shared memory: tables, then two stages of PSI[c][MIX_NP] + RAD[lam][MIX_NP].  Wide
// dipole coefficients per group slot are field contracted at staging:
//   length gauge   DA = coef_k                (acc += DA r_a psi_s)
//   velocity gauge DA = i coef_k ldiff_k, DB = i coef_k   (acc += DA psi_s/(2 r_a) + DB W_a[s])
// with coef_k = field . dcoef(:, k), zero below 1e-30 (the skip of src/kernels.f90:145).
// ---------------------------------------------------------------------------------
template <typename R> struct MixSmem {
    cplx<R> *da, *db, *stage;
    R *wcoef;
    int *wsrc, *wptr, *dsrc, *del;
};

template <typename R>
__device__ __forceinline__ MixSmem<R> mix_layout(unsigned char *raw, const TiledPlan<R> &pl)
{
    MixSmem<R> s;
    s.da = reinterpret_cast<cplx<R> *>(raw);
    s.db = s.da + (size_t)max(pl.nwd, 1) * MIX_GROUP;
    s.stage = s.db + (size_t)max(pl.nwd, 1) * MIX_GROUP;
    s.wcoef = reinterpret_cast<R *>(s.stage + 2 * (size_t)(pl.nc + pl.nlam) * MIX_NP);
    s.wsrc = reinterpret_cast<int *>(s.wcoef + (size_t)pl.nwide * MIX_GROUP);
    s.wptr = s.wsrc + pl.nwide;
    s.dsrc = s.wptr + pl.ng * pl.nlam + 1;
    s.del = s.dsrc + pl.nwd;
    return s;
}

template <typename R>
__device__ __forceinline__ void mix_prefetch(const cplx<R> *psi, const cplx<R> *rad, size_t nn, int nc, int nlam,
                                             size_t p0, cplx<R> *dst)
{
    const int rows = nc + nlam;
    for (int idx = threadIdx.x; idx < rows * MIX_NP; idx += blockDim.x) {
        const int q = idx % MIX_NP, row = idx / MIX_NP;
        const size_t p = p0 + q;
        const bool ok = p < nn;
        const cplx<R> *src = row < nc ? psi + (ok ? p : 0) + nn * row : rad + (ok ? p : 0) + nn * (row - nc);
        cp_async<sizeof(cplx<R>)>(dst + idx, src, ok ? (int)sizeof(cplx<R>) : 0);
    }
    cp_async_commit();
}

template <typename R, bool VEL>
__global__ void __launch_bounds__(512, 1)
hpsi_mix_kernel(const DeviceTables<R> t, const TiledPlan<R> pl, const cplx<R> *__restrict__ psi,
                cplx<R> *__restrict__ out, const cplx<R> *__restrict__ w1, const cplx<R> *__restrict__ w2,
                R f0, R f1, R f2, cplx<R> beta, cplx<R> gamma)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = pl.n, nc = pl.nc, nlam = pl.nlam;
    const MixSmem<R> S = mix_layout<R>(smem_raw, pl);
    const size_t nn = (size_t)n * n;
    const size_t ntiles = (nn + MIX_NP - 1) / MIX_NP;
    const int stage_elems = (nc + nlam) * MIX_NP;

    size_t tile = blockIdx.x;
    if (tile < ntiles) mix_prefetch<R>(psi, t.rad, nn, nc, nlam, tile * MIX_NP, S.stage);
    for (int idx = threadIdx.x; idx < pl.nwd * MIX_GROUP; idx += blockDim.x) {
        const int kk = pl.dwedge[idx];
        cplx<R> a = mk<R>(0, 0), b = mk<R>(0, 0);
        if (kk >= 0) {
            const cplx<R> *dk = t.dcoef + 3 * (size_t)kk;
            cplx<R> v = cscale<R>(f0, dk[0]);
            v = rfma<R>(f1, dk[1], v);
            v = rfma<R>(f2, dk[2], v);
            if (sqrt(cabs2<R>(v)) < (R)1e-30) v = mk<R>(0, 0);
            if (VEL) {
                b = mk<R>(-v.y, v.x);                 // i coef
                a = cscale<R>(t.ldiff[kk], b);        // i coef ldiff
            } else {
                a = v;
            }
        }
        S.da[idx] = a;
        S.db[idx] = b;
    }
    for (int k = threadIdx.x; k < pl.nwide * MIX_GROUP; k += blockDim.x) S.wcoef[k] = pl.wcoef[k];
    for (int k = threadIdx.x; k < pl.nwide; k += blockDim.x) S.wsrc[k] = pl.wsrc[k] * MIX_NP;
    for (int k = threadIdx.x; k <= pl.ng * nlam; k += blockDim.x) S.wptr[k] = pl.wptr[k];
    for (int k = threadIdx.x; k < pl.nwd; k += blockDim.x) {
        S.dsrc[k] = pl.dwsrc[k] * MIX_NP;
        S.del[k] = pl.dwel[k];
    }

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
        const int buf = it & 1;
        const cplx<R> *PSI = S.stage + buf * stage_elems;
        const cplx<R> *RAD = PSI + (size_t)nc * MIX_NP;
        const size_t next = tile + gridDim.x;
        if (next < ntiles) {
            mix_prefetch<R>(psi, t.rad, nn, nc, nlam, next * MIX_NP, S.stage + (buf ^ 1) * stage_elems);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const size_t p0 = tile * MIX_NP;
        const int np = (int)min((size_t)MIX_NP, nn - p0);
        const bool v0 = lane < np, v1 = lane + 32 < np;
        const size_t pa = p0 + lane, pb = p0 + lane + 32;
        for (int g = warp; g < pl.ng; g += nwarps) {
            int ch[MIX_GROUP];
            cplx<R> o0[MIX_GROUP], o1[MIX_GROUP], a0[MIX_GROUP], a1[MIX_GROUP];
#pragma unroll
            for (int d = 0; d < MIX_GROUP; ++d) {   // radial part: loads issued now, used at the end
                ch[d] = __ldg(pl.gch + g * MIX_GROUP + d);
                o0[d] = (v0 && ch[d] >= 0) ? out[pa + nn * ch[d]] : mk<R>(0, 0);
                o1[d] = (v1 && ch[d] >= 0) ? out[pb + nn * ch[d]] : mk<R>(0, 0);
                a0[d] = mk<R>(0, 0);
                a1[d] = mk<R>(0, 0);
            }
            const int *wp = S.wptr + g * nlam;
            for (int lam = 0; lam < nlam; ++lam) {
                const int k0 = wp[lam], k1 = wp[lam + 1];
                if (k0 == k1) continue;
                cplx<R> t0[MIX_GROUP], t1[MIX_GROUP];
#pragma unroll
                for (int d = 0; d < MIX_GROUP; ++d) { t0[d] = mk<R>(0, 0); t1[d] = mk<R>(0, 0); }
#pragma unroll 2
                for (int k = k0; k < k1; ++k) {
                    const int off = S.wsrc[k];
                    const cplx<R> x0 = PSI[off + lane], x1 = PSI[off + lane + 32];
                    const R *cf = S.wcoef + k * MIX_GROUP;
#pragma unroll
                    for (int d = 0; d < MIX_GROUP; ++d) {
                        const R w = cf[d];
                        t0[d] = rfma<R>(w, x0, t0[d]);
                        t1[d] = rfma<R>(w, x1, t1[d]);
                    }
                }
                const cplx<R> r0 = RAD[lam * MIX_NP + lane], r1 = RAD[lam * MIX_NP + lane + 32];
#pragma unroll
                for (int d = 0; d < MIX_GROUP; ++d) {
                    a0[d] = cfma<R>(r0, t0[d], a0[d]);
                    a1[d] = cfma<R>(r1, t1[d], a1[d]);
                }
            }
            const int k0 = __ldg(pl.dwptr + g), k1 = __ldg(pl.dwptr + g + 1);
            if (k0 < k1) {
                const int ia = (int)(pa % n), ja = (int)(pa / n), ib = (int)(pb % n), jb = (int)(pb / n);
                const cplx<R> *rt = VEL ? t.hinv : t.r;   // r (length) or 1/(2r) (velocity)
                const cplx<R> ra1 = v0 ? ldg<R>(rt + ia) : mk<R>(0, 0), ra2 = v0 ? ldg<R>(rt + ja) : mk<R>(0, 0);
                const cplx<R> rb1 = v1 ? ldg<R>(rt + ib) : mk<R>(0, 0), rb2 = v1 ? ldg<R>(rt + jb) : mk<R>(0, 0);
                for (int k = k0; k < k1; ++k) {
                    const int off = S.dsrc[k];
                    const bool first = S.del[k] == 1;
                    const cplx<R> y0 = cmul<R>(first ? ra1 : ra2, PSI[off + lane]);
                    const cplx<R> y1 = cmul<R>(first ? rb1 : rb2, PSI[off + lane + 32]);
                    const cplx<R> *da = S.da + k * MIX_GROUP;
#pragma unroll
                    for (int d = 0; d < MIX_GROUP; ++d) {
                        a0[d] = cfma<R>(da[d], y0, a0[d]);
                        a1[d] = cfma<R>(da[d], y1, a1[d]);
                    }
                    if (VEL) {
                        const int s = off / MIX_NP;
                        const cplx<R> *wsrc = first ? w1 : w2;
                        const cplx<R> wa = v0 ? wsrc[pa + nn * s] : mk<R>(0, 0);
                        const cplx<R> wb = v1 ? wsrc[pb + nn * s] : mk<R>(0, 0);
                        const cplx<R> *db = S.db + k * MIX_GROUP;
#pragma unroll
                        for (int d = 0; d < MIX_GROUP; ++d) {
                            a0[d] = cfma<R>(db[d], wa, a0[d]);
                            a1[d] = cfma<R>(db[d], wb, a1[d]);
                        }
                    }
                }
            }
#pragma unroll
            for (int d = 0; d < MIX_GROUP; ++d) {
                if (ch[d] < 0) continue;
                if (v0) out[pa + nn * ch[d]] = cfma<R>(gamma, cadd<R>(a0[d], o0[d]), cmul<R>(beta, PSI[ch[d] * MIX_NP + lane]));
                if (v1) out[pb + nn * ch[d]] = cfma<R>(gamma, cadd<R>(a1[d], o1[d]), cmul<R>(beta, PSI[ch[d] * MIX_NP + lane + 32]));
            }
        }
        __syncthreads();   // the stage buffer is refilled two tiles later
    }
}

template <typename R> size_t radial_smem(bool vel, int blkmax)
{
    return sizeof(cplx<R>) * (2 * (size_t)RAD_STRIDE * RAD_STRIDE + (size_t)RAD_TMAX * RAD_STRIDE +
                              (vel ? 4 : 2) * (size_t)blkmax);
}

template <typename R> size_t mix_smem(int nc, int nlam, int ng, int nwide, int nwd)
{
    const size_t c = sizeof(cplx<R>) * (2 * (size_t)(nc + nlam) * MIX_NP + 2 * (size_t)std::max(nwd, 1) * MIX_GROUP);
    const size_t r = sizeof(R) * (size_t)nwide * MIX_GROUP;
    const size_t i = sizeof(int) * ((size_t)nwide + (size_t)ng * nlam + 1 + 2 * (size_t)nwd);
    return c + r + i + 64;
}

// True when a batch of fb.count > 1 instances can run as one launch per kernel (banded
// kinetic kernel and generated mixing kernel); otherwise the caller applies the
// instances one at a time.
template <typename R> bool tiled_batchable(he_operator *h, const void *psi, int velocity)
{
    return h->path == 1 && band_usable<R>(band_plan<R>(h), psi) && h->mixpath == 1 &&
           jit_mix_prepare(h, (sizeof(R) == 8 ? 0 : 2) + (velocity ? 1 : 0)) == HE_OK;
}

template <typename R>
int launch_hpsi_tiled(he_operator *h, const DeviceTables<R> &t, const TiledPlan<R> &pl, cplx<R> *coef,
                      cplx<R> *w1, cplx<R> *w2, const cplx<R> *psi, cplx<R> *out, const FieldBatch &fb, int velocity,
                      cplx<R> beta, cplx<R> gamma, cudaStream_t stream)
{
    (void)coef;
    const double *field = fb.f[0];
    if (fb.count > 1 && !tiled_batchable<R>(h, psi, velocity))
        return he_fail(HE_ERR_UNSUPPORTED, "batched apply needs the banded and generated kernels", __FILE__, __LINE__);
    const R f0 = (R)field[0], f1 = (R)field[1], f2 = (R)field[2];
    const R a2 = (R)(field[0] * field[0] + field[1] * field[1] + field[2] * field[2]);
    const KineticPlan<R> &kp = kinetic_plan<R>(h);
    if (h->path == 1 && band_usable<R>(band_plan<R>(h), psi)) {
        const int s = launch_band<R>(h, t, band_plan<R>(h), psi, out, w1, w2, fb, velocity, stream);
        if (s) return s;
    } else if ((h->path == 1 || h->path == 3) && kinetic_usable<R>(kp, psi)) {
        const int s = launch_kinetic<R>(h, t, kp, psi, out, w1, w2, a2, velocity, stream);
        if (s) return s;
    } else {
        const dim3 rgrid(pl.ntile * pl.ntile, (pl.nc + RAD_CH - 1) / RAD_CH);
        const int blkmax = h->plan.blkmax;
        const size_t rs = radial_smem<R>(velocity, blkmax);
#define HE_RADIAL(V, S)                                                                                  \
    do {                                                                                                 \
        auto kern = hpsi_radial_kernel<R, V, S>;                                                         \
        HE_CUDA_TRY(he_smem_limit(reinterpret_cast<const void *>(kern), rs));                            \
        kern<<<rgrid, RAD_THREADS, rs, stream>>>(t, pl, psi, out, w1, w2, a2, blkmax);                   \
    } while (0)
        if (velocity) { if (t.diag_separable) HE_RADIAL(true, true); else HE_RADIAL(true, false); }
        else { if (t.diag_separable) HE_RADIAL(false, true); else HE_RADIAL(false, false); }
#undef HE_RADIAL
        HE_CUDA_TRY(cudaGetLastError());
    }
    if (h->mixpath == 1 && jit_mix_prepare(h, (sizeof(R) == 8 ? 0 : 2) + (velocity ? 1 : 0)) == HE_OK)
        return launch_mix_jit<R>(h, t, psi, out, w1, w2, fb, velocity, beta, gamma, stream);
    const size_t nn = (size_t)pl.n * pl.n;
    const size_t ms = mix_smem<R>(pl.nc, pl.nlam, pl.ng, pl.nwide, pl.nwd);
    const size_t ntiles = (nn + MIX_NP - 1) / MIX_NP;
    const int per_sm = std::max<int>(1, (int)((227 * 1024) / (ms + 1024)));
    const unsigned blocks = (unsigned)std::min<size_t>(ntiles, (size_t)148 * per_sm);
    const int threads = 32 * std::min(16, std::max(1, pl.ng));
    if (velocity) {
        HE_CUDA_TRY(he_smem_limit(reinterpret_cast<const void *>(hpsi_mix_kernel<R, true>), ms));
        hpsi_mix_kernel<R, true><<<blocks, threads, ms, stream>>>(t, pl, psi, out, w1, w2, f0, f1, f2, beta, gamma);
    } else {
        HE_CUDA_TRY(he_smem_limit(reinterpret_cast<const void *>(hpsi_mix_kernel<R, false>), ms));
        hpsi_mix_kernel<R, false><<<blocks, threads, ms, stream>>>(t, pl, psi, out, w1, w2, f0, f1, f2, beta, gamma);
    }
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

template bool tiled_batchable<double>(he_operator *, const void *, int);
template bool tiled_batchable<float>(he_operator *, const void *, int);
template int launch_hpsi_tiled<double>(he_operator *, const DeviceTables<double> &, const TiledPlan<double> &,
                                       double2 *, double2 *, double2 *, const double2 *, double2 *, const FieldBatch &,
                                       int, double2, double2, cudaStream_t);
template int launch_hpsi_tiled<float>(he_operator *, const DeviceTables<float> &, const TiledPlan<float> &, float2 *,
                                      float2 *, float2 *, const float2 *, float2 *, const FieldBatch &, int, float2,
                                      float2, cudaStream_t);

// Both kernels must fit in shared memory (one CTA per SM) in complex128.
bool tiled_fits(const he_plan_host &P, int nc, int nd)
{
    (void)nd;
    return mix_smem<double>(nc, P.nlam, P.ng, (int)P.wsrc.size(), (int)P.dwsrc.size()) <= 200 * 1024 &&
           radial_smem<double>(true, P.blkmax) <= 200 * 1024;
}

}  // namespace he
