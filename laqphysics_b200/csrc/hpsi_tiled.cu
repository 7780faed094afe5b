// Tiled two-electron H·psi for sm_100a (the production path; hamiltonian.cu keeps the
// generic one-thread-per-output kernel for tables this plan cannot express).
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
//   hpsi_mix_kernel     per point, all channels of 128 points staged in shared memory:
//                       Coulomb multipoles sum_lam rad_lam sum_c' V_lam[c,c'] psi_c' and the
//                       dipole couplings, register-blocked over MIX_GROUP output channels
//                       that share source channels ("wide edges"), then the epilogue
//                       out = beta psi + gamma (H psi).
//
// Each kernel reads psi once from DRAM; the radial result travels through `out`.
#include <algorithm>
#include <complex>
#include <cstring>
#include <map>
#include <numeric>
#include <set>

#include "common.cuh"
#include "hpsi_tiled.cuh"
#include "operator.cuh"

namespace he {

constexpr int RAD_THREADS = 256;
constexpr int RAD_STRIDE = RAD_TMAX + 1;   // odd row stride (in complex elements): conflict-free columns

template <typename R> __device__ __forceinline__ cplx<R> cmul_sel(bool real, cplx<R> a, cplx<R> x, cplx<R> acc)
{
    return real ? rfma<R>(a.x, x, acc) : cfma<R>(a, x, acc);
}

// Element e: nodes [s, s + m - 1], m = estart[e+1] - s + 1 (last element: n - s).
__device__ __forceinline__ int elem_size(const int *estart, int e, int ne, int n)
{
    return e + 1 < ne ? estart[e + 1] - estart[e] + 1 : n - estart[e];
}

// ---------------------------------------------------------------------------------
// Radial stencil kernel.  grid = (ntile * ntile, nc); one channel-tile per CTA.
// Smem: PS[(rows+1) x RAD_STRIDE] staged psi (owned + right bridge), OS owned output,
// W1S/W2S owned B-stencil results (velocity gauge only).
// ---------------------------------------------------------------------------------
template <typename R, bool VEL, bool SEP>
__global__ void __launch_bounds__(RAD_THREADS)
hpsi_radial_kernel(const DeviceTables<R> t, const TiledPlan<R> pl, const cplx<R> *__restrict__ psi,
                   cplx<R> *__restrict__ out, cplx<R> *__restrict__ w1, cplx<R> *__restrict__ w2, R a2)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R> *PS = reinterpret_cast<cplx<R> *>(smem_raw);
    cplx<R> *OS = PS + RAD_STRIDE * RAD_STRIDE;
    cplx<R> *W1S = OS + RAD_TMAX * RAD_STRIDE;
    cplx<R> *W2S = W1S + RAD_TMAX * RAD_STRIDE;

    const int n = pl.n, ne = pl.ne;
    const int ti = blockIdx.x % pl.ntile, tj = blockIdx.x / pl.ntile, c = blockIdx.y;
    const int ea = pl.tstart[ti], eb = pl.tstart[ti + 1];
    const int fa = pl.tstart[tj], fb = pl.tstart[tj + 1];
    const int r0 = pl.estart[ea], r1 = pl.estart[eb];          // owned rows [r0, r1)
    const int c0 = pl.estart[fa], c1 = pl.estart[fb];          // owned cols [c0, c1)
    const int rs = min(r1 + 1, n) - r0, cs = min(c1 + 1, n) - c0;   // staged extents (+ right bridge)
    const int ro = r1 - r0, co = c1 - c0;
    const size_t nn = (size_t)n * n;
    const cplx<R> *pc = psi + nn * c;

    // stage psi rows [r0, r0+rs) x cols [c0, c0+cs): lanes along rows (contiguous i)
    for (int idx = threadIdx.x; idx < rs * cs; idx += blockDim.x) {
        const int a = idx % rs, b = idx / rs;
        PS[a * RAD_STRIDE + b] = pc[(size_t)(r0 + a) + (size_t)n * (c0 + b)];
    }
    __syncthreads();

    // ---- phase 1: electron 1 (rows); item = (owned column, element, row chunk) -------
    {
        int nitems = 0;
        for (int e = ea; e < eb; ++e) {
            const int own = (e + 1 < ne ? pl.estart[e + 1] : n) - pl.estart[e];
            nitems += co * ((own + RAD_CHUNK - 1) / RAD_CHUNK);
        }
        for (int item = threadIdx.x; item < nitems; item += blockDim.x) {
            int rest = item, e = ea;
            for (; e < eb; ++e) {
                const int own = (e + 1 < ne ? pl.estart[e + 1] : n) - pl.estart[e];
                const int cnt = co * ((own + RAD_CHUNK - 1) / RAD_CHUNK);
                if (rest < cnt) break;
                rest -= cnt;
            }
            const int col = rest % co, chunk = rest / co;
            const int s = pl.estart[e], m = elem_size(pl.estart, e, ne, n);
            const int own = (e + 1 < ne ? pl.estart[e + 1] : n) - s;
            const int a0 = chunk * RAD_CHUNK, na = min(RAD_CHUNK, own - a0);
            const cplx<R> *blk = pl.blocks + pl.eoff[e];
            const cplx<R> *bbl = pl.bblocks + pl.eoff[e];
            const bool real = pl.ereal[e];
            cplx<R> acc[RAD_CHUNK], accb[RAD_CHUNK];
#pragma unroll
            for (int q = 0; q < RAD_CHUNK; ++q) { acc[q] = mk<R>(0, 0); accb[q] = mk<R>(0, 0); }
            for (int b = 0; b < m; ++b) {
                const cplx<R> x = PS[(s - r0 + b) * RAD_STRIDE + col];
#pragma unroll
                for (int q = 0; q < RAD_CHUNK; ++q) {
                    if (q < na) {
                        acc[q] = cmul_sel<R>(real, blk[(a0 + q) * m + b], x, acc[q]);
                        if (VEL) accb[q] = cmul_sel<R>(real, bbl[(a0 + q) * m + b], x, accb[q]);
                    }
                }
            }
            if (a0 == 0 && e > 0) {   // left bridge row s: the previous element's part
                const int sp = pl.estart[e - 1], mp = elem_size(pl.estart, e - 1, ne, n);
                const cplx<R> *bp = pl.blocks + pl.eoff[e - 1] + (size_t)(mp - 1) * mp;
                const cplx<R> *bq = pl.bblocks + pl.eoff[e - 1] + (size_t)(mp - 1) * mp;
                const bool rp = pl.ereal[e - 1];
                for (int b = 0; b < mp - 1; ++b) {
                    const int row = sp + b;
                    const cplx<R> x = row >= r0 ? PS[(row - r0) * RAD_STRIDE + col]
                                                : pc[(size_t)row + (size_t)n * (c0 + col)];
                    acc[0] = cmul_sel<R>(rp, bp[b], x, acc[0]);
                    if (VEL) accb[0] = cmul_sel<R>(rp, bq[b], x, accb[0]);
                }
            }
#pragma unroll
            for (int q = 0; q < RAD_CHUNK; ++q) {
                if (q < na) {
                    const int row = s - r0 + a0 + q;
                    OS[row * RAD_STRIDE + col] = acc[q];
                    if (VEL) W1S[row * RAD_STRIDE + col] = accb[q];
                }
            }
        }
    }
    __syncthreads();

    // ---- phase 2: electron 2 (columns); item = (owned row, element, column chunk) -----
    {
        int nitems = 0;
        for (int f = fa; f < fb; ++f) {
            const int own = (f + 1 < ne ? pl.estart[f + 1] : n) - pl.estart[f];
            nitems += ro * ((own + RAD_CHUNK - 1) / RAD_CHUNK);
        }
        for (int item = threadIdx.x; item < nitems; item += blockDim.x) {
            int rest = item, f = fa;
            for (; f < fb; ++f) {
                const int own = (f + 1 < ne ? pl.estart[f + 1] : n) - pl.estart[f];
                const int cnt = ro * ((own + RAD_CHUNK - 1) / RAD_CHUNK);
                if (rest < cnt) break;
                rest -= cnt;
            }
            const int row = rest % ro, chunk = rest / ro;
            const int s = pl.estart[f], m = elem_size(pl.estart, f, ne, n);
            const int own = (f + 1 < ne ? pl.estart[f + 1] : n) - s;
            const int a0 = chunk * RAD_CHUNK, na = min(RAD_CHUNK, own - a0);
            const cplx<R> *blk = pl.blocks + pl.eoff[f];
            const cplx<R> *bbl = pl.bblocks + pl.eoff[f];
            const bool real = pl.ereal[f];
            cplx<R> acc[RAD_CHUNK], accb[RAD_CHUNK];
#pragma unroll
            for (int q = 0; q < RAD_CHUNK; ++q) { acc[q] = mk<R>(0, 0); accb[q] = mk<R>(0, 0); }
            for (int b = 0; b < m; ++b) {
                const cplx<R> x = PS[row * RAD_STRIDE + (s - c0 + b)];
#pragma unroll
                for (int q = 0; q < RAD_CHUNK; ++q) {
                    if (q < na) {
                        acc[q] = cmul_sel<R>(real, blk[(a0 + q) * m + b], x, acc[q]);
                        if (VEL) accb[q] = cmul_sel<R>(real, bbl[(a0 + q) * m + b], x, accb[q]);
                    }
                }
            }
            if (a0 == 0 && f > 0) {
                const int sp = pl.estart[f - 1], mp = elem_size(pl.estart, f - 1, ne, n);
                const cplx<R> *bp = pl.blocks + pl.eoff[f - 1] + (size_t)(mp - 1) * mp;
                const cplx<R> *bq = pl.bblocks + pl.eoff[f - 1] + (size_t)(mp - 1) * mp;
                const bool rp = pl.ereal[f - 1];
                for (int b = 0; b < mp - 1; ++b) {
                    const int colg = sp + b;
                    const cplx<R> x = colg >= c0 ? PS[row * RAD_STRIDE + (colg - c0)]
                                                 : pc[(size_t)(r0 + row) + (size_t)n * colg];
                    acc[0] = cmul_sel<R>(rp, bp[b], x, acc[0]);
                    if (VEL) accb[0] = cmul_sel<R>(rp, bq[b], x, accb[0]);
                }
            }
#pragma unroll
            for (int q = 0; q < RAD_CHUNK; ++q) {
                if (q < na) {
                    const int col = s - c0 + a0 + q;
                    OS[row * RAD_STRIDE + col] = cadd<R>(OS[row * RAD_STRIDE + col], acc[q]);
                    if (VEL) W2S[row * RAD_STRIDE + col] = accb[q];
                }
            }
        }
    }
    __syncthreads();

    // ---- epilogue: diagonal (+|A|^2), write the radial part (and W) ------------------
    for (int idx = threadIdx.x; idx < ro * co; idx += blockDim.x) {
        const int a = idx % ro, b = idx / ro;
        const int i = r0 + a, j = c0 + b;
        const size_t p = (size_t)i + (size_t)n * j;
        const cplx<R> x = PS[a * RAD_STRIDE + b];
        cplx<R> d = SEP ? cadd<R>(ldg<R>(t.d1 + i + (size_t)n * c), ldg<R>(t.d2 + j + (size_t)n * c))
                        : ldg<R>(t.diag + p + nn * c);
        cplx<R> v = cfma<R>(d, x, OS[a * RAD_STRIDE + b]);
        if (VEL) {
            v = rfma<R>(a2, x, v);
            w1[p + nn * c] = W1S[a * RAD_STRIDE + b];
            w2[p + nn * c] = W2S[a * RAD_STRIDE + b];
        }
        out[p + nn * c] = v;
    }
}

// ---------------------------------------------------------------------------------
// Field contraction of the dipole edges: coef_k = field . dcoef(:, k), zero below 1e-30
// (the skip of src/kernels.f90:145).
// ---------------------------------------------------------------------------------
template <typename R>
__global__ void contract_field_kernel(const cplx<R> *__restrict__ dcoef, int nd, R f0, R f1, R f2,
                                      cplx<R> *__restrict__ coef)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nd; k += gridDim.x * blockDim.x) {
        cplx<R> v = cscale<R>(f0, dcoef[3 * k]);
        v = rfma<R>(f1, dcoef[3 * k + 1], v);
        v = rfma<R>(f2, dcoef[3 * k + 2], v);
        if (sqrt(cabs2<R>(v)) < (R)1e-30) v = mk<R>(0, 0);
        coef[k] = v;
    }
}

// ---------------------------------------------------------------------------------
// Channel-mixing kernel.  CTA = NP consecutive flattened points p = i + n j, all
// channels staged as PSI[c][NP]; multipoles staged as RAD[lam][NP].  A warp task is
// (32 points, one output group); accumulators live in registers.
// ---------------------------------------------------------------------------------
template <typename R, bool VEL, int NP>
__global__ void __launch_bounds__(256)
hpsi_mix_kernel(const DeviceTables<R> t, const TiledPlan<R> pl, const cplx<R> *__restrict__ psi,
                cplx<R> *__restrict__ out, const cplx<R> *__restrict__ w1, const cplx<R> *__restrict__ w2,
                const cplx<R> *__restrict__ coef, cplx<R> beta, cplx<R> gamma)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cplx<R> *PSI = reinterpret_cast<cplx<R> *>(smem_raw);
    cplx<R> *RAD = PSI + (size_t)pl.nc * NP;
    const int n = pl.n, nc = pl.nc, nlam = pl.nlam;
    const size_t nn = (size_t)n * n;
    const size_t p0 = (size_t)blockIdx.x * NP;
    const int np = (int)min((size_t)NP, nn - p0);

    for (int idx = threadIdx.x; idx < nc * NP; idx += blockDim.x) {
        const int q = idx % NP, cc = idx / NP;
        PSI[idx] = q < np ? psi[p0 + q + nn * cc] : mk<R>(0, 0);
    }
    for (int idx = threadIdx.x; idx < nlam * NP; idx += blockDim.x) {
        const int q = idx % NP, lam = idx / NP;
        RAD[idx] = q < np ? ldg<R>(t.rad + p0 + q + nn * lam) : mk<R>(0, 0);
    }
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
        // Coulomb multipoles, grouped by lambda
        for (int lam = 0; lam < nlam; ++lam) {
            const int k0 = __ldg(pl.wptr + g * nlam + lam), k1 = __ldg(pl.wptr + g * nlam + lam + 1);
            if (k0 == k1) continue;
            cplx<R> tsum[MIX_GROUP];
#pragma unroll
            for (int d = 0; d < MIX_GROUP; ++d) tsum[d] = mk<R>(0, 0);
            for (int k = k0; k < k1; ++k) {
                const cplx<R> x = PSI[__ldg(pl.wsrc + k) * NP + q];
#pragma unroll
                for (int d = 0; d < MIX_GROUP; ++d) tsum[d] = rfma<R>(__ldg(pl.wcoef + k * MIX_GROUP + d), x, tsum[d]);
            }
            const cplx<R> rl = RAD[lam * NP + q];
#pragma unroll
            for (int d = 0; d < MIX_GROUP; ++d) acc[d] = cfma<R>(rl, tsum[d], acc[d]);
        }
        // dipole couplings
        const int k0 = __ldg(pl.dwptr + g), k1 = __ldg(pl.dwptr + g + 1);
        if (k0 < k1 && valid) {
            const int i = (int)(p % n), j = (int)(p / n);
            for (int k = k0; k < k1; ++k) {
                const int s = __ldg(pl.dwsrc + k);
                const int el = __ldg(pl.dwel + k);
                const int a = el == 1 ? i : j;
                const cplx<R> x = PSI[s * NP + q];
                if (!VEL) {
                    const cplx<R> y = cmul<R>(ldg<R>(t.r + a), x);
#pragma unroll
                    for (int d = 0; d < MIX_GROUP; ++d) {
                        const int kk = __ldg(pl.dwedge + k * MIX_GROUP + d);
                        if (kk >= 0) acc[d] = cfma<R>(ldg<R>(coef + kk), y, acc[d]);
                    }
                } else {
                    const cplx<R> w = (el == 1 ? w1 : w2)[p + nn * s];
                    const cplx<R> hx = cmul<R>(ldg<R>(t.hinv + a), x);
#pragma unroll
                    for (int d = 0; d < MIX_GROUP; ++d) {
                        const int kk = __ldg(pl.dwedge + k * MIX_GROUP + d);
                        if (kk >= 0) {
                            const cplx<R> part = rfma<R>(__ldg(t.ldiff + kk), hx, w);
                            const cplx<R> cf = ldg<R>(coef + kk);
                            acc[d] = cfma<R>(mk<R>(-cf.y, cf.x), part, acc[d]);   // i coef part
                        }
                    }
                }
            }
        }
        if (valid) {
#pragma unroll
            for (int d = 0; d < MIX_GROUP; ++d)
                if (ch[d] >= 0) out[p + nn * ch[d]] = cfma<R>(gamma, acc[d], cmul<R>(beta, PSI[ch[d] * NP + q]));
        }
    }
}

template <typename R> static size_t radial_smem(bool vel)
{
    return sizeof(cplx<R>) * ((size_t)RAD_STRIDE * RAD_STRIDE + (vel ? 3 : 1) * (size_t)RAD_TMAX * RAD_STRIDE);
}

template <typename R> static size_t mix_smem(int nc, int nlam, int np)
{
    return sizeof(cplx<R>) * (size_t)(nc + nlam) * np;
}

template <typename R>
int launch_hpsi_tiled(he_operator *h, const DeviceTables<R> &t, const TiledPlan<R> &pl, cplx<R> *coef,
                      cplx<R> *w1, cplx<R> *w2, const cplx<R> *psi, cplx<R> *out, const double *field, int velocity,
                      cplx<R> beta, cplx<R> gamma, cudaStream_t stream)
{
    const R f0 = (R)field[0], f1 = (R)field[1], f2 = (R)field[2];
    const R a2 = (R)(field[0] * field[0] + field[1] * field[1] + field[2] * field[2]);
    if (t.nd > 0) contract_field_kernel<R><<<1, 256, 0, stream>>>(t.dcoef, t.nd, f0, f1, f2, coef);
    const dim3 rgrid(pl.ntile * pl.ntile, pl.nc);
    const size_t rs = radial_smem<R>(velocity);
#define HE_RADIAL(V, S)                                                                                  \
    do {                                                                                                 \
        auto kern = hpsi_radial_kernel<R, V, S>;                                                         \
        HE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rs));   \
        kern<<<rgrid, RAD_THREADS, rs, stream>>>(t, pl, psi, out, w1, w2, a2);                           \
    } while (0)
    if (velocity) { if (t.diag_separable) HE_RADIAL(true, true); else HE_RADIAL(true, false); }
    else { if (t.diag_separable) HE_RADIAL(false, true); else HE_RADIAL(false, false); }
#undef HE_RADIAL
    HE_CUDA_TRY(cudaGetLastError());
    const size_t nn = (size_t)pl.n * pl.n;
    const size_t limit = 200 * 1024;
#define HE_MIX(V, NP)                                                                                    \
    do {                                                                                                 \
        auto kern = hpsi_mix_kernel<R, V, NP>;                                                           \
        const size_t ms = mix_smem<R>(pl.nc, pl.nlam, NP);                                               \
        HE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ms));   \
        kern<<<(unsigned)((nn + NP - 1) / NP), 256, ms, stream>>>(t, pl, psi, out, w1, w2, coef, beta, gamma); \
    } while (0)
    const int np = mix_smem<R>(pl.nc, pl.nlam, 128) <= limit ? 128 : mix_smem<R>(pl.nc, pl.nlam, 64) <= limit ? 64 : 32;
    if (velocity) {
        if (np == 128) HE_MIX(true, 128); else if (np == 64) HE_MIX(true, 64); else HE_MIX(true, 32);
    } else {
        if (np == 128) HE_MIX(false, 128); else if (np == 64) HE_MIX(false, 64); else HE_MIX(false, 32);
    }
#undef HE_MIX
    HE_CUDA_TRY(cudaGetLastError());
    (void)h;
    return HE_OK;
}

template int launch_hpsi_tiled<double>(he_operator *, const DeviceTables<double> &, const TiledPlan<double> &,
                                       double2 *, double2 *, double2 *, const double2 *, double2 *, const double *,
                                       int, double2, double2, cudaStream_t);
template int launch_hpsi_tiled<float>(he_operator *, const DeviceTables<float> &, const TiledPlan<float> &, float2 *,
                                      float2 *, float2 *, const float2 *, float2 *, const double *, int, float2,
                                      float2, cudaStream_t);

bool tiled_fits(int nc, int nlam, size_t elem)
{
    return elem * (size_t)(nc + nlam) * 32 <= 200 * 1024;
}

}  // namespace he

// =====================================================================================
// Host planning
// =====================================================================================
namespace {

struct UnionFind {
    std::vector<int> p;
    explicit UnionFind(int n) : p(n) { std::iota(p.begin(), p.end(), 0); }
    int find(int x) { while (p[x] != x) x = p[x] = p[p[x]]; return x; }
    void join(int a, int b) { p[find(a)] = find(b); }
};

}  // namespace

// Build the tiled plan from the reference's tables.  Returns false (and the generic
// kernel is used) when the kinetic matrix is not block banded by elements, an element
// is too large for a shared-memory tile, or a Coulomb coefficient is not real.
bool he_build_plan(he_plan_host &P, int n, int nc, const int *ptr, const int *col, const double *tv, int nv,
                   const int *vptr, const int *vc, const int *vl, const double *vcoef, int nlam, int nd,
                   const int *dptr, const int *dc, const int *de, const double *r)
{
    using he::MIX_GROUP;
    P = he_plan_host();
    // --- elements from the first column of each row ---------------------------------
    std::vector<int> first(n), last(n);
    std::set<int> starts;
    for (int i = 0; i < n; ++i) {
        if (ptr[i + 1] == ptr[i]) return false;
        int lo = n, hi = -1;
        for (int k = ptr[i]; k < ptr[i + 1]; ++k) { lo = std::min(lo, col[k]); hi = std::max(hi, col[k]); }
        first[i] = lo; last[i] = hi;
        starts.insert(lo);
    }
    if (!starts.count(0)) return false;
    P.estart.assign(starts.begin(), starts.end());
    const int ne = (int)P.estart.size();
    P.estart.push_back(n);
    P.ne = ne;
    auto esize = [&](int e) { return e + 1 < ne ? P.estart[e + 1] - P.estart[e] + 1 : n - P.estart[e]; };
    // every entry of row i (owned by element e) must lie in element e, or in e-1 for a bridge row
    for (int e = 0; e < ne; ++e) {
        const int s = P.estart[e], m = esize(e);
        if (m > he::RAD_TMAX + 1 || m < 2) return false;
        const int own_end = e + 1 < ne ? P.estart[e + 1] : n;
        for (int i = s; i < own_end; ++i) {
            const int lo_ok = (i == s && e > 0) ? P.estart[e - 1] : s;
            if (first[i] < lo_ok || last[i] > s + m - 1) return false;
        }
    }
    // --- dense element blocks of T and of B = T (r_b - r_a) ---------------------------
    P.eoff.assign(ne + 1, 0);
    for (int e = 0; e < ne; ++e) P.eoff[e + 1] = P.eoff[e] + esize(e) * esize(e);
    P.blocks.assign(2 * (size_t)P.eoff[ne], 0.0);
    P.bblocks.assign(2 * (size_t)P.eoff[ne], 0.0);
    P.ereal.assign(ne, 1);
    for (int e = 0; e < ne; ++e) {
        const int s = P.estart[e], m = esize(e);
        P.maxm = std::max(P.maxm, m);
        for (int a = 0; a < m; ++a) {
            const int i = s + a;
            for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
                const int b = col[k] - s;
                if (b < 0 || b >= m) continue;   // the previous element's part of a bridge row
                const std::complex<double> T(tv[2 * k], tv[2 * k + 1]);
                const std::complex<double> ra(r[2 * i], r[2 * i + 1]), rb(r[2 * col[k]], r[2 * col[k] + 1]);
                const std::complex<double> B = T * (rb - ra);
                const size_t o = 2 * ((size_t)P.eoff[e] + (size_t)a * m + b);
                P.blocks[o] = T.real(); P.blocks[o + 1] = T.imag();
                P.bblocks[o] = B.real(); P.bblocks[o + 1] = B.imag();
                if (T.imag() != 0.0 || B.imag() != 0.0) P.ereal[e] = 0;
            }
        }
    }
    // --- radial tiles: up to RAD_ELEMS elements and RAD_TMAX owned nodes --------------
    P.tstart.push_back(0);
    for (int e = 0; e < ne;) {
        int cnt = 0, own = 0, f = e;
        while (f < ne && cnt < he::RAD_ELEMS) {
            const int o = (f + 1 < ne ? P.estart[f + 1] : n) - P.estart[f];
            if (own + o > he::RAD_TMAX) break;
            own += o; ++cnt; ++f;
        }
        if (cnt == 0) return false;
        e = f;
        P.tstart.push_back(e);
    }
    P.ntile = (int)P.tstart.size() - 1;
    // --- output groups: channels of one Coulomb component with shared sources ---------
    for (int k = 0; k < nv; ++k)
        if (vcoef[2 * k + 1] != 0.0) return false;
    P.nlam = nlam;
    UnionFind uf(nc);
    std::vector<std::set<std::pair<int, int>>> src(nc);
    for (int c = 0; c < nc; ++c)
        for (int k = vptr[c]; k < vptr[c + 1]; ++k) { uf.join(c, vc[k]); src[c].insert({vc[k], vl[k]}); }
    std::vector<int> assigned(nc, 0);
    std::vector<std::vector<int>> groups;
    for (int c = 0; c < nc; ++c) {
        if (assigned[c]) continue;
        std::vector<int> grp{c};
        assigned[c] = 1;
        while ((int)grp.size() < MIX_GROUP) {
            int best = -1, score = -1;
            for (int x = 0; x < nc; ++x) {
                if (assigned[x] || uf.find(x) != uf.find(c)) continue;
                int s = 0;
                for (auto &e : src[x]) s += (int)src[c].count(e);
                if (s > score) { score = s; best = x; }
            }
            if (best < 0) break;
            grp.push_back(best);
            assigned[best] = 1;
        }
        groups.push_back(grp);
    }
    P.ng = (int)groups.size();
    P.gch.assign((size_t)P.ng * MIX_GROUP, -1);
    P.wptr.assign((size_t)P.ng * nlam + 1, 0);
    P.dwptr.assign(P.ng + 1, 0);
    for (int g = 0; g < P.ng; ++g) {
        const auto &grp = groups[g];
        for (int d = 0; d < (int)grp.size(); ++d) P.gch[(size_t)g * MIX_GROUP + d] = grp[d];
        for (int lam = 0; lam < nlam; ++lam) {
            std::map<int, std::vector<double>> wide;
            for (int d = 0; d < (int)grp.size(); ++d)
                for (int k = vptr[grp[d]]; k < vptr[grp[d] + 1]; ++k)
                    if (vl[k] == lam) {
                        auto &w = wide[vc[k]];
                        if (w.empty()) w.assign(MIX_GROUP, 0.0);
                        w[d] += vcoef[2 * k];
                    }
            for (auto &kv : wide) {
                P.wsrc.push_back(kv.first);
                P.wcoef.insert(P.wcoef.end(), kv.second.begin(), kv.second.end());
            }
            P.wptr[(size_t)g * nlam + lam + 1] = (int)P.wsrc.size();
        }
        // dipole edges keyed by (source, electron); repeated keys of one channel open a new slot
        std::vector<std::pair<std::pair<int, int>, std::vector<int>>> dw;
        for (int d = 0; d < (int)grp.size(); ++d)
            for (int k = dptr[grp[d]]; k < dptr[grp[d] + 1]; ++k) {
                bool placed = false;
                for (auto &slot : dw)
                    if (slot.first == std::make_pair(dc[k], de[k]) && slot.second[d] < 0) {
                        slot.second[d] = k; placed = true; break;
                    }
                if (!placed) {
                    std::vector<int> v(MIX_GROUP, -1);
                    v[d] = k;
                    dw.push_back({{dc[k], de[k]}, v});
                }
            }
        for (auto &slot : dw) {
            P.dwsrc.push_back(slot.first.first);
            P.dwel.push_back(slot.first.second);
            P.dwedge.insert(P.dwedge.end(), slot.second.begin(), slot.second.end());
        }
        P.dwptr[g + 1] = (int)P.dwsrc.size();
    }
    (void)nd;
    P.ok = true;
    return true;
}

// ---------------------------------------------------------------------------------
// Planner inspection (host only, no GPU needed): build the plan for a set of tables
// and copy its arrays out, so the tile and group layout can be checked on the CPU.
// ---------------------------------------------------------------------------------
extern "C" void *he_plan_build(int n, int nc, const int *ptr, const int *col, const double *tv, int nv,
                               const int *vptr, const int *vc, const int *vl, const double *vcoef, int nlam, int nd,
                               const int *dptr, const int *dc, const int *de, const double *r)
{
    he_plan_host *P = new he_plan_host();
    he_build_plan(*P, n, nc, ptr, col, tv, nv, vptr, vc, vl, vcoef, nlam, nd, dptr, dc, de, r);
    return P;
}

extern "C" void he_plan_free(void *plan) { delete static_cast<he_plan_host *>(plan); }

// which: 0 estart, 1 tstart, 2 eoff, 3 ereal, 4 gch, 5 wptr, 6 wsrc, 7 dwptr, 8 dwsrc, 9 dwel, 10 dwedge,
//        20 blocks (interleaved complex), 21 bblocks, 22 wcoef, 30 scalars {ok, ne, ntile, ng, nlam, maxm}.
// Returns the element count; copies when dst != NULL.
extern "C" long long he_plan_array(void *plan, int which, void *dst)
{
    const he_plan_host &P = *static_cast<he_plan_host *>(plan);
    const std::vector<int> *vi = nullptr;
    const std::vector<double> *vd = nullptr;
    switch (which) {
    case 0: vi = &P.estart; break;
    case 1: vi = &P.tstart; break;
    case 2: vi = &P.eoff; break;
    case 3: vi = &P.ereal; break;
    case 4: vi = &P.gch; break;
    case 5: vi = &P.wptr; break;
    case 6: vi = &P.wsrc; break;
    case 7: vi = &P.dwptr; break;
    case 8: vi = &P.dwsrc; break;
    case 9: vi = &P.dwel; break;
    case 10: vi = &P.dwedge; break;
    case 20: vd = &P.blocks; break;
    case 21: vd = &P.bblocks; break;
    case 22: vd = &P.wcoef; break;
    case 30: {
        const int s[6] = {P.ok, P.ne, P.ntile, P.ng, P.nlam, P.maxm};
        if (dst) memcpy(dst, s, sizeof(s));
        return 6;
    }
    default: return -1;
    }
    if (vi) { if (dst) memcpy(dst, vi->data(), vi->size() * sizeof(int)); return (long long)vi->size(); }
    if (dst) memcpy(dst, vd->data(), vd->size() * sizeof(double));
    return (long long)vd->size();
}
