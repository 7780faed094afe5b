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
//   hpsi_mix_kernel     per point, all channels of NP points staged in shared memory:
//                       Coulomb multipoles sum_lam rad_lam sum_c' V_lam[c,c'] psi_c' and the
//                       dipole couplings, register-blocked over MIX_GROUP output channels
//                       that share source channels ("wide edges"), then the epilogue
//                       out = beta psi + gamma (H psi).
//
// psi is read once from DRAM by each kernel; the radial result travels through `out`.
// Every table an inner loop touches (element blocks, wide edges, dipole edges) is
// staged in shared memory first, so the loops issue no global loads.
#include <algorithm>

#include "common.cuh"
#include "hpsi_tiled.cuh"
#include "operator.cuh"

namespace he {

constexpr int RAD_THREADS = 256;
constexpr int RAD_STRIDE = RAD_TMAX + 1;   // odd row stride (complex elements): conflict-free column reads

template <typename R> __device__ __forceinline__ cplx<R> cmul_sel(bool real, cplx<R> a, cplx<R> x, cplx<R> acc)
{
    return real ? rfma<R>(a.x, x, acc) : cfma<R>(a, x, acc);
}

// Per-axis description of a radial tile, built in shared memory by the CTA.
struct AxisTile {
    int ga, gb;                          // element range
    int count;                           // gb - ga
    int s[RAD_ELEMS], m[RAD_ELEMS], own[RAD_ELEMS], real[RAD_ELEMS];
    int off[RAD_ELEMS];                  // offset of the element's T block in the staged blocks
    int items[RAD_ELEMS + 1];            // prefix sums of work items (lines x chunks)
    int prev, prev_m, prev_real, prev_off;   // previous element (bridge row), -1 if none
};

// Stage the element blocks of one axis: previous element's last row, then full blocks.
// Returns the number of complex entries written for one matrix kind (T or B).
template <typename R>
__device__ void stage_axis(const TiledPlan<R> &pl, AxisTile &ax, int ga, int gb, int lines, cplx<R> *dst,
                           cplx<R> *dstB, bool vel)
{
    const int n = pl.n, ne = pl.ne;
    if (threadIdx.x == 0) {
        ax.ga = ga; ax.gb = gb; ax.count = gb - ga;
        int off = 0;
        ax.prev = ga > 0 ? ga - 1 : -1;
        if (ga > 0) {
            const int e = ga - 1;
            ax.prev_m = e + 1 < ne ? pl.estart[e + 1] - pl.estart[e] + 1 : n - pl.estart[e];
            ax.prev_real = pl.ereal[e];
            ax.prev_off = 0;
            off = ax.prev_m;
        }
        ax.items[0] = 0;
        for (int k = 0; k < ax.count; ++k) {
            const int e = ga + k;
            ax.s[k] = pl.estart[e];
            ax.m[k] = e + 1 < ne ? pl.estart[e + 1] - pl.estart[e] + 1 : n - pl.estart[e];
            ax.own[k] = (e + 1 < ne ? pl.estart[e + 1] : n) - pl.estart[e];
            ax.real[k] = pl.ereal[e];
            ax.off[k] = off;
            off += ax.m[k] * ax.m[k];
            ax.items[k + 1] = ax.items[k] + lines * ((ax.own[k] + RAD_CHUNK - 1) / RAD_CHUNK);
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

// One direction of the radial stencil on the staged tile.  ROWS = electron 1 (lines are
// owned columns, element index runs along rows), else electron 2.
template <typename R, bool VEL, bool ROWS>
__device__ void radial_phase(const AxisTile &ax, const cplx<R> *BLK, const cplx<R> *BLKB, const cplx<R> *PS,
                             cplx<R> *OS, int lines, int base, int r0, int c0, int n, const cplx<R> *pc,
                             cplx<R> *wout, size_t nn, int c)
{
    const int nitems = ax.items[ax.count];
    for (int item = threadIdx.x; item < nitems; item += blockDim.x) {
        int k = 0;
        while (k + 1 < ax.count && item >= ax.items[k + 1]) ++k;
        const int rest = item - ax.items[k];
        const int line = rest % lines, chunk = rest / lines;
        const int s = ax.s[k], m = ax.m[k];
        const int a0 = chunk * RAD_CHUNK, na = min(RAD_CHUNK, ax.own[k] - a0);
        const cplx<R> *blk = BLK + ax.off[k], *bbl = BLKB + ax.off[k];
        const bool real = ax.real[k];
        cplx<R> acc[RAD_CHUNK], accb[RAD_CHUNK];
#pragma unroll
        for (int q = 0; q < RAD_CHUNK; ++q) { acc[q] = mk<R>(0, 0); accb[q] = mk<R>(0, 0); }
        for (int b = 0; b < m; ++b) {
            const int node = s - base + b;
            const cplx<R> x = ROWS ? PS[node * RAD_STRIDE + line] : PS[line * RAD_STRIDE + node];
#pragma unroll
            for (int q = 0; q < RAD_CHUNK; ++q) {
                if (q < na) {
                    acc[q] = cmul_sel<R>(real, blk[(a0 + q) * m + b], x, acc[q]);
                    if (VEL) accb[q] = cmul_sel<R>(real, bbl[(a0 + q) * m + b], x, accb[q]);
                }
            }
        }
        if (a0 == 0 && (k > 0 || ax.prev >= 0)) {   // bridge row s: the previous element's part
            const cplx<R> *bp, *bq;
            int mp, sp;
            bool rp;
            if (k > 0) {
                mp = ax.m[k - 1]; sp = ax.s[k - 1]; rp = ax.real[k - 1];
                bp = BLK + ax.off[k - 1] + (mp - 1) * mp; bq = BLKB + ax.off[k - 1] + (mp - 1) * mp;
            } else {
                mp = ax.prev_m; sp = s - (mp - 1); rp = ax.prev_real;
                bp = BLK + ax.prev_off; bq = BLKB + ax.prev_off;
            }
            for (int b = 0; b < mp - 1; ++b) {
                const int node = sp + b;   // global index along this axis
                cplx<R> x;
                if (node >= base) x = ROWS ? PS[(node - base) * RAD_STRIDE + line] : PS[line * RAD_STRIDE + node - base];
                else x = ROWS ? pc[(size_t)node + (size_t)n * (c0 + line)] : pc[(size_t)(r0 + line) + (size_t)n * node];
                acc[0] = cmul_sel<R>(rp, bp[b], x, acc[0]);
                if (VEL) accb[0] = cmul_sel<R>(rp, bq[b], x, accb[0]);
            }
        }
#pragma unroll
        for (int q = 0; q < RAD_CHUNK; ++q) {
            if (q < na) {
                const int node = s - base + a0 + q;
                const int row = ROWS ? node : line, col = ROWS ? line : node;
                if (ROWS) OS[row * RAD_STRIDE + col] = acc[q];
                else OS[row * RAD_STRIDE + col] = cadd<R>(OS[row * RAD_STRIDE + col], acc[q]);
                if (VEL) wout[(size_t)(r0 + row) + (size_t)n * (c0 + col) + nn * c] = accb[q];
            }
        }
    }
}

// ---------------------------------------------------------------------------------
// Radial stencil kernel.  grid = (ntile * ntile, nc); one channel-tile per CTA.
// ---------------------------------------------------------------------------------
template <typename R, bool VEL, bool SEP>
__global__ void __launch_bounds__(RAD_THREADS, 2)
hpsi_radial_kernel(const DeviceTables<R> t, const TiledPlan<R> pl, const cplx<R> *__restrict__ psi,
                   cplx<R> *__restrict__ out, cplx<R> *__restrict__ w1, cplx<R> *__restrict__ w2, R a2, int blkmax)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R> *PS = reinterpret_cast<cplx<R> *>(smem_raw);
    cplx<R> *OS = PS + RAD_STRIDE * RAD_STRIDE;
    cplx<R> *B0 = OS + RAD_TMAX * RAD_STRIDE;        // electron-1 blocks (T), then B if VEL
    cplx<R> *B0B = B0 + blkmax;
    cplx<R> *B1 = B0 + (VEL ? 2 : 1) * blkmax;       // electron-2 blocks
    cplx<R> *B1B = B1 + blkmax;
    __shared__ AxisTile ax0, ax1;

    const int n = pl.n;
    const int ti = blockIdx.x % pl.ntile, tj = blockIdx.x / pl.ntile, c = blockIdx.y;
    const int ea = pl.tstart[ti], eb = pl.tstart[ti + 1];
    const int fa = pl.tstart[tj], fb = pl.tstart[tj + 1];
    const int r0 = pl.estart[ea], r1 = pl.estart[eb];          // owned rows [r0, r1)
    const int c0 = pl.estart[fa], c1 = pl.estart[fb];          // owned cols [c0, c1)
    const int rs = min(r1 + 1, n) - r0, cs = min(c1 + 1, n) - c0;   // staged extents (+ right bridge)
    const int ro = r1 - r0, co = c1 - c0;
    const size_t nn = (size_t)n * n;
    const cplx<R> *pc = psi + nn * c;

    for (int idx = threadIdx.x; idx < rs * cs; idx += blockDim.x) {
        const int a = idx % rs, b = idx / rs;
        PS[a * RAD_STRIDE + b] = pc[(size_t)(r0 + a) + (size_t)n * (c0 + b)];
    }
    stage_axis<R>(pl, ax0, ea, eb, co, B0, B0B, VEL);
    stage_axis<R>(pl, ax1, fa, fb, ro, B1, B1B, VEL);
    __syncthreads();
    radial_phase<R, VEL, true>(ax0, B0, B0B, PS, OS, co, r0, r0, c0, n, pc, w1, nn, c);
    __syncthreads();
    radial_phase<R, VEL, false>(ax1, B1, B1B, PS, OS, ro, c0, r0, c0, n, pc, w2, nn, c);
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
}

// ---------------------------------------------------------------------------------
// Channel-mixing kernel.  CTA = NP consecutive flattened points p = i + n j.
// Shared memory: PSI[c][NP], RAD[lam][NP], wide Coulomb edges (source offset, MIX_GROUP
// coefficients), group x lam offsets, wide dipole edges and the field-contracted
// dipole coefficients coef_k = field . dcoef(:, k) (zero below 1e-30, the skip of
// src/kernels.f90:145).  A warp task is (32 points, one output group).
// ---------------------------------------------------------------------------------
template <typename R> struct MixSmem {
    cplx<R> *psi, *rad, *coef;
    R *wcoef, *ldiff;
    int *wsrc, *wptr, *dsrc, *del, *dedge;
};

template <typename R>
__device__ __forceinline__ MixSmem<R> mix_layout(unsigned char *raw, const TiledPlan<R> &pl, int nd, int np)
{
    MixSmem<R> s;
    s.psi = reinterpret_cast<cplx<R> *>(raw);
    s.rad = s.psi + (size_t)pl.nc * np;
    s.coef = s.rad + (size_t)pl.nlam * np;
    s.wcoef = reinterpret_cast<R *>(s.coef + max(nd, 1));
    s.ldiff = s.wcoef + (size_t)pl.nwide * MIX_GROUP;
    s.wsrc = reinterpret_cast<int *>(s.ldiff + max(nd, 1));
    s.wptr = s.wsrc + pl.nwide;
    s.dsrc = s.wptr + pl.ng * pl.nlam + 1;
    s.del = s.dsrc + pl.nwd;
    s.dedge = s.del + pl.nwd;
    return s;
}

template <typename R, bool VEL, int NP>
__global__ void __launch_bounds__(256)
hpsi_mix_kernel(const DeviceTables<R> t, const TiledPlan<R> pl, const cplx<R> *__restrict__ psi,
                cplx<R> *__restrict__ out, const cplx<R> *__restrict__ w1, const cplx<R> *__restrict__ w2,
                R f0, R f1, R f2, cplx<R> beta, cplx<R> gamma)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = pl.n, nc = pl.nc, nlam = pl.nlam, nd = t.nd;
    const MixSmem<R> S = mix_layout<R>(smem_raw, pl, nd, NP);
    const size_t nn = (size_t)n * n;
    const size_t p0 = (size_t)blockIdx.x * NP;
    const int np = (int)min((size_t)NP, nn - p0);

    for (int idx = threadIdx.x; idx < nc * NP; idx += blockDim.x) {
        const int q = idx % NP, cc = idx / NP;
        S.psi[idx] = q < np ? psi[p0 + q + nn * cc] : mk<R>(0, 0);
    }
    for (int idx = threadIdx.x; idx < nlam * NP; idx += blockDim.x) {
        const int q = idx % NP, lam = idx / NP;
        S.rad[idx] = q < np ? ldg<R>(t.rad + p0 + q + nn * lam) : mk<R>(0, 0);
    }
    for (int k = threadIdx.x; k < nd; k += blockDim.x) {
        const cplx<R> *dk = t.dcoef + 3 * (size_t)k;
        cplx<R> v = cscale<R>(f0, dk[0]);
        v = rfma<R>(f1, dk[1], v);
        v = rfma<R>(f2, dk[2], v);
        if (sqrt(cabs2<R>(v)) < (R)1e-30) v = mk<R>(0, 0);
        S.coef[k] = v;
        S.ldiff[k] = t.ldiff[k];
    }
    for (int k = threadIdx.x; k < pl.nwide * MIX_GROUP; k += blockDim.x) S.wcoef[k] = pl.wcoef[k];
    for (int k = threadIdx.x; k < pl.nwide; k += blockDim.x) S.wsrc[k] = pl.wsrc[k] * NP;
    for (int k = threadIdx.x; k <= pl.ng * nlam; k += blockDim.x) S.wptr[k] = pl.wptr[k];
    for (int k = threadIdx.x; k < pl.nwd; k += blockDim.x) {
        S.dsrc[k] = pl.dwsrc[k];
        S.del[k] = pl.dwel[k];
    }
    for (int k = threadIdx.x; k < pl.nwd * MIX_GROUP; k += blockDim.x) S.dedge[k] = pl.dwedge[k];
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    constexpr int QUARTERS = NP / 32;
    for (int task = warp; task < pl.ng * QUARTERS; task += nwarps) {
        const int g = task / QUARTERS, quarter = task % QUARTERS;
        const int q = quarter * 32 + lane;
        const bool valid = q < np;
        const size_t p = p0 + q;
        int ch[MIX_GROUP];
        cplx<R> acc[MIX_GROUP];
#pragma unroll
        for (int d = 0; d < MIX_GROUP; ++d) {
            ch[d] = __ldg(pl.gch + g * MIX_GROUP + d);
            acc[d] = (valid && ch[d] >= 0) ? out[p + nn * ch[d]] : mk<R>(0, 0);
        }
        const int *wp = S.wptr + g * nlam;
        for (int lam = 0; lam < nlam; ++lam) {
            const int k0 = wp[lam], k1 = wp[lam + 1];
            if (k0 == k1) continue;
            cplx<R> tsum[MIX_GROUP];
#pragma unroll
            for (int d = 0; d < MIX_GROUP; ++d) tsum[d] = mk<R>(0, 0);
#pragma unroll 2
            for (int k = k0; k < k1; ++k) {
                const cplx<R> x = S.psi[S.wsrc[k] + q];
                const R *cf = S.wcoef + k * MIX_GROUP;
#pragma unroll
                for (int d = 0; d < MIX_GROUP; ++d) tsum[d] = rfma<R>(cf[d], x, tsum[d]);
            }
            const cplx<R> rl = S.rad[lam * NP + q];
#pragma unroll
            for (int d = 0; d < MIX_GROUP; ++d) acc[d] = cfma<R>(rl, tsum[d], acc[d]);
        }
        const int k0 = __ldg(pl.dwptr + g), k1 = __ldg(pl.dwptr + g + 1);
        if (k0 < k1 && valid) {
            const int i = (int)(p % n), j = (int)(p / n);
            const cplx<R> r1 = ldg<R>(t.r + i), r2 = ldg<R>(t.r + j);
            const cplx<R> h1 = ldg<R>(t.hinv + i), h2 = ldg<R>(t.hinv + j);
            for (int k = k0; k < k1; ++k) {
                const int s = S.dsrc[k];
                const bool first = S.del[k] == 1;
                const cplx<R> x = S.psi[s * NP + q];
                if (!VEL) {
                    const cplx<R> y = cmul<R>(first ? r1 : r2, x);
#pragma unroll
                    for (int d = 0; d < MIX_GROUP; ++d) {
                        const int kk = S.dedge[k * MIX_GROUP + d];
                        if (kk >= 0) acc[d] = cfma<R>(S.coef[kk], y, acc[d]);
                    }
                } else {
                    const cplx<R> w = (first ? w1 : w2)[p + nn * s];
                    const cplx<R> hx = cmul<R>(first ? h1 : h2, x);
#pragma unroll
                    for (int d = 0; d < MIX_GROUP; ++d) {
                        const int kk = S.dedge[k * MIX_GROUP + d];
                        if (kk >= 0) {
                            const cplx<R> part = rfma<R>(S.ldiff[kk], hx, w);
                            const cplx<R> cf = S.coef[kk];
                            acc[d] = cfma<R>(mk<R>(-cf.y, cf.x), part, acc[d]);   // i coef part
                        }
                    }
                }
            }
        }
        if (valid) {
#pragma unroll
            for (int d = 0; d < MIX_GROUP; ++d)
                if (ch[d] >= 0) out[p + nn * ch[d]] = cfma<R>(gamma, acc[d], cmul<R>(beta, S.psi[ch[d] * NP + q]));
        }
    }
}

template <typename R> size_t radial_smem(bool vel, int blkmax)
{
    return sizeof(cplx<R>) * ((size_t)RAD_STRIDE * RAD_STRIDE + (size_t)RAD_TMAX * RAD_STRIDE +
                              (vel ? 4 : 2) * (size_t)blkmax);
}

template <typename R> size_t mix_smem(const TiledPlan<R> &pl, int nd, int np)
{
    const size_t c = sizeof(cplx<R>) * ((size_t)(pl.nc + pl.nlam) * np + std::max(nd, 1));
    const size_t r = sizeof(R) * ((size_t)pl.nwide * MIX_GROUP + std::max(nd, 1));
    const size_t i = sizeof(int) * ((size_t)pl.nwide + pl.ng * pl.nlam + 1 + pl.nwd * (2 + MIX_GROUP));
    return c + r + i + 64;
}

template <typename R>
int launch_hpsi_tiled(he_operator *h, const DeviceTables<R> &t, const TiledPlan<R> &pl, cplx<R> *coef,
                      cplx<R> *w1, cplx<R> *w2, const cplx<R> *psi, cplx<R> *out, const double *field, int velocity,
                      cplx<R> beta, cplx<R> gamma, cudaStream_t stream)
{
    (void)coef;
    const R f0 = (R)field[0], f1 = (R)field[1], f2 = (R)field[2];
    const R a2 = (R)(field[0] * field[0] + field[1] * field[1] + field[2] * field[2]);
    const dim3 rgrid(pl.ntile * pl.ntile, pl.nc);
    const int blkmax = h->plan.blkmax;
    const size_t rs = radial_smem<R>(velocity, blkmax);
#define HE_RADIAL(V, S)                                                                                  \
    do {                                                                                                 \
        auto kern = hpsi_radial_kernel<R, V, S>;                                                         \
        HE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rs));   \
        kern<<<rgrid, RAD_THREADS, rs, stream>>>(t, pl, psi, out, w1, w2, a2, blkmax);                   \
    } while (0)
    if (velocity) { if (t.diag_separable) HE_RADIAL(true, true); else HE_RADIAL(true, false); }
    else { if (t.diag_separable) HE_RADIAL(false, true); else HE_RADIAL(false, false); }
#undef HE_RADIAL
    HE_CUDA_TRY(cudaGetLastError());
    const size_t nn = (size_t)pl.n * pl.n;
    const size_t limit = 110 * 1024;   // two CTAs per SM
    const int np = (sizeof(R) == 4 && mix_smem<R>(pl, t.nd, 128) <= limit) ? 128
                 : mix_smem<R>(pl, t.nd, 64) <= limit ? 64 : 32;
#define HE_MIX(V, NP)                                                                                    \
    do {                                                                                                 \
        auto kern = hpsi_mix_kernel<R, V, NP>;                                                           \
        const size_t ms = mix_smem<R>(pl, t.nd, NP);                                                     \
        HE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ms));   \
        kern<<<(unsigned)((nn + NP - 1) / NP), 256, ms, stream>>>(t, pl, psi, out, w1, w2, f0, f1, f2, beta, gamma); \
    } while (0)
    if (velocity) {
        if (np == 128) HE_MIX(true, 128); else if (np == 64) HE_MIX(true, 64); else HE_MIX(true, 32);
    } else {
        if (np == 128) HE_MIX(false, 128); else if (np == 64) HE_MIX(false, 64); else HE_MIX(false, 32);
    }
#undef HE_MIX
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

template int launch_hpsi_tiled<double>(he_operator *, const DeviceTables<double> &, const TiledPlan<double> &,
                                       double2 *, double2 *, double2 *, const double2 *, double2 *, const double *,
                                       int, double2, double2, cudaStream_t);
template int launch_hpsi_tiled<float>(he_operator *, const DeviceTables<float> &, const TiledPlan<float> &, float2 *,
                                      float2 *, float2 *, const float2 *, float2 *, const double *, int, float2,
                                      float2, cudaStream_t);

// The mixing kernel must fit two CTAs of 32 points per SM in complex128.
bool tiled_fits(const he_plan_host &P, int nc, int nd)
{
    TiledPlan<double> pl{};
    pl.nc = nc; pl.nlam = P.nlam; pl.ng = P.ng; pl.nwide = (int)P.wsrc.size(); pl.nwd = (int)P.dwsrc.size();
    return mix_smem<double>(pl, nd, 32) <= 110 * 1024 && radial_smem<double>(true, P.blkmax) <= 110 * 1024;
}

}  // namespace he
