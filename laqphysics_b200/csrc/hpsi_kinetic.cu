// Kinetic energy of both electrons, the diagonal and |A|^2 of H·psi on TMA-staged tiles
// (src/kernels.f90:132-143 and :170; in the velocity gauge also the commutator stencils
// W_e = B_e psi, B = T (r_b - r_a), of :153-168, which the channel-mixing kernel consumes).
//
// Work is a list of (row tile, column tile, channel) items, split evenly over a
// persistent grid of two CTAs per SM.  For each item one TMA copy (cp.async.bulk.tensor,
// 3-D map over psi(re/im, r1, r2·channel)) brings the staged box into shared memory;
// the copy of the next item is in flight while the current one is computed (two stages,
// one mbarrier each, one __syncthreads per item).
//
// Thread (row lane, slot) owns up to KIN_NA outputs psi(i, s_f + a0 + q): lanes run along
// r1, so every global store is coalesced and both directions accumulate in registers:
//   along r2   acc[q] += sum_b T_f[a0+q][b] psi(i, s_f + b)       (slot-uniform T, broadcast)
//   along r1   acc[q] += sum_b T_e[a_i][b] psi(s_e + b, s_f+a0+q) (per-lane T row)
// plus the bridge rows/columns, whose previous-element nodes are part of the staged box.
#include <cudaTypedefs.h>

#include <mutex>

#include "common.cuh"
#include "hpsi_kinetic.cuh"
#include "operator.cuh"

namespace he {

constexpr int KIN_WAIT_LIMIT = 1 << 21;          // try_wait rounds before a stage counts as lost
constexpr unsigned KIN_WAIT_HINT_NS = 2000;      // suspend hint of one try_wait round

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(KIN_WAIT_HINT_NS)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity)
{
    for (int k = 0; k < KIN_WAIT_LIMIT; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Tiled TMA load of one box into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

template <typename R> __device__ __forceinline__ int elem_size(const KineticPlan<R> &kp, int e)
{
    return (e + 1 < kp.ne ? kp.estart[e + 1] + 1 : kp.n) - kp.estart[e];
}

template <typename R> struct pair_t;
template <> struct pair_t<double> { using type = double2; };
template <> struct pair_t<float> { using type = float2; };
template <typename R> __device__ __forceinline__ typename pair_t<R>::type ldg_pair(const R *p)
{
    return __ldg(reinterpret_cast<const typename pair_t<R>::type *>(p));
}

// acc[q] += X[a0+q][b] x for q < na; k = index of X^T[b][a0] in the padded planes (even,
// so each pair of coefficients is one vector load; the loads are uniform over the warp).
template <typename R, bool REAL>
__device__ __forceinline__ void r2_tap(const R *__restrict__ xre, const R *__restrict__ xim, int k, cplx<R> x, int na,
                                       cplx<R> (&acc)[KIN_NA])
{
#pragma unroll
    for (int q = 0; q < KIN_NA; q += 2) {
        if (q < na) {
            const auto tr = ldg_pair<R>(xre + k + q);
            if (REAL) {
                acc[q] = rfma<R>(tr.x, x, acc[q]);
                if (q + 1 < na) acc[q + 1] = rfma<R>(tr.y, x, acc[q + 1]);
            } else {
                const auto ti = ldg_pair<R>(xim + k + q);
                acc[q] = cfma<R>(mk<R>(tr.x, ti.x), x, acc[q]);
                if (q + 1 < na) acc[q + 1] = cfma<R>(mk<R>(tr.y, ti.y), x, acc[q + 1]);
            }
        }
    }
}

// Along r2 over the nodes of element f (size M at compile time, or m when M == 0):
// acc[q] += sum_b X_f[a0+q][b] S(s_f + b, i); `col` points at S(s_f, i).
template <typename R, bool REAL, int M>
__device__ __forceinline__ void r2_element(const R *xre, const R *xim, int koff, int m, int a0, int na,
                                           const cplx<R> *col, int pitch, cplx<R> (&acc)[KIN_NA])
{
    if constexpr (M > 0) {
        constexpr int MP = M + (M & 1);
#pragma unroll
        for (int b = 0; b < M; ++b) r2_tap<R, REAL>(xre, xim, koff + b * MP + a0, col[b * pitch], na, acc);
    } else {
        const int mp = m + (m & 1);
        for (int b = 0; b < m; ++b) r2_tap<R, REAL>(xre, xim, koff + b * mp + a0, col[b * pitch], na, acc);
    }
}

template <typename R>
__device__ __forceinline__ void along_r2(const KineticPlan<R> &kp, const R *__restrict__ xre, const R *__restrict__ xim,
                                         const cplx<R> *S, int pitch, int il, int y0, int f, int a0, int na,
                                         cplx<R> (&acc)[KIN_NA])
{
    const int sf = kp.estart[f], mf = elem_size(kp, f), koff = kp.koff[f];
    const cplx<R> *col = S + (sf - y0) * pitch + il;
    const bool real = kp.ereal[f];
    switch (real ? mf : -mf) {   // slot-uniform: the common FE sizes get exact unrolls
    case 9: r2_element<R, true, 9>(xre, xim, koff, mf, a0, na, col, pitch, acc); break;
    case 10: r2_element<R, true, 10>(xre, xim, koff, mf, a0, na, col, pitch, acc); break;
    case -9: r2_element<R, false, 9>(xre, xim, koff, mf, a0, na, col, pitch, acc); break;
    case -10: r2_element<R, false, 10>(xre, xim, koff, mf, a0, na, col, pitch, acc); break;
    default:
        if (real) r2_element<R, true, 0>(xre, xim, koff, mf, a0, na, col, pitch, acc);
        else r2_element<R, false, 0>(xre, xim, koff, mf, a0, na, col, pitch, acc);
    }
    if (a0 == 0 && f > 0) {   // bridge column s_f: the previous element's last row
        const int fp = f - 1, sp = kp.estart[fp], mp = sf - sp + 1, mpp = mp + (mp & 1), kf = kp.koff[fp];
        const cplx<R> *colp = S + (sp - y0) * pitch + il;
        const bool rp = kp.ereal[fp];
        cplx<R> s = acc[0];
        for (int b = 0; b < mp - 1; ++b) {
            const int k = kf + b * mpp + (mp - 1);
            const cplx<R> x = colp[b * pitch];
            s = rp ? rfma<R>(__ldg(xre + k), x, s) : cfma<R>(mk<R>(__ldg(xre + k), __ldg(xim + k)), x, s);
        }
        acc[0] = s;
    }
}

// Along r1 for row i = s_e + a_i over element e's own nodes: acc[q] += sum_b X_e[a_i][b]
// S(cq0 + q, s_e + b); `rows` points at S(cq0, s_e).  The coefficient row sits in registers.
template <typename R, bool REAL, int M>
__device__ __forceinline__ void r1_row(const R *__restrict__ xre, const R *__restrict__ xim, int koff, int m, int ai,
                                       int na, const cplx<R> *rows, int pitch, cplx<R> (&acc)[KIN_NA])
{
    if constexpr (M > 0) {
        constexpr int MP = M + (M & 1);
        R tr[M], ti[M];
#pragma unroll
        for (int b = 0; b < M; ++b) {
            tr[b] = __ldg(xre + koff + b * MP + ai);
            ti[b] = REAL ? (R)0 : __ldg(xim + koff + b * MP + ai);
        }
#pragma unroll
        for (int q = 0; q < KIN_NA; ++q) {
            if (q < na) {
                const cplx<R> *rq = rows + q * pitch;
                cplx<R> s = acc[q];
#pragma unroll
                for (int b = 0; b < M; ++b) s = REAL ? rfma<R>(tr[b], rq[b], s) : cfma<R>(mk<R>(tr[b], ti[b]), rq[b], s);
                acc[q] = s;
            }
        }
    } else {
        const int mp = m + (m & 1);
        for (int b = 0; b < m; ++b) {
            const R tr = __ldg(xre + koff + b * mp + ai), ti = REAL ? (R)0 : __ldg(xim + koff + b * mp + ai);
#pragma unroll
            for (int q = 0; q < KIN_NA; ++q)
                if (q < na) acc[q] = REAL ? rfma<R>(tr, rows[q * pitch + b], acc[q])
                                          : cfma<R>(mk<R>(tr, ti), rows[q * pitch + b], acc[q]);
        }
    }
}

// Along r1 for row i.  The bridge-row part (i = s_e: the previous element's last row) is
// added here only when `bridge` is set (the velocity-gauge W1 pass); the kinetic pass
// takes it from the per-item bridge partials instead.
template <typename R>
__device__ __forceinline__ void along_r1(const KineticPlan<R> &kp, const R *__restrict__ xre, const R *__restrict__ xim,
                                         const cplx<R> *S, int pitch, int i, int x0, int cq0, int y0, int na, bool bridge,
                                         cplx<R> (&acc)[KIN_NA])
{
    const int e = kp.nodeelem[i], se = kp.estart[e], me = elem_size(kp, e), ai = i - se, koff = kp.koff[e];
    const cplx<R> *rows = S + (cq0 - y0) * pitch + (se - x0);
    const bool real = kp.ereal[e];
    switch (real ? me : -me) {
    case 9: r1_row<R, true, 9>(xre, xim, koff, me, ai, na, rows, pitch, acc); break;
    case 10: r1_row<R, true, 10>(xre, xim, koff, me, ai, na, rows, pitch, acc); break;
    default:
        if (real) r1_row<R, true, 0>(xre, xim, koff, me, ai, na, rows, pitch, acc);
        else r1_row<R, false, 0>(xre, xim, koff, me, ai, na, rows, pitch, acc);
    }
    if (bridge && ai == 0 && e > 0) {
        const int ep = e - 1, sp = kp.estart[ep], mp = se - sp + 1, mpp = mp + (mp & 1), kf = kp.koff[ep];
        const cplx<R> *rp = S + (cq0 - y0) * pitch + (sp - x0);
        const bool real_p = kp.ereal[ep];
        for (int b = 0; b < mp - 1; ++b) {
            const int k = kf + b * mpp + (mp - 1);
            const cplx<R> tv = mk<R>(__ldg(xre + k), real_p ? (R)0 : __ldg(xim + k));
#pragma unroll
            for (int q = 0; q < KIN_NA; ++q)
                if (q < na) acc[q] = real_p ? rfma<R>(tv.x, rp[q * pitch + b], acc[q])
                                            : cfma<R>(tv, rp[q * pitch + b], acc[q]);
        }
    }
}

template <typename R, bool VEL, bool SEP>
__global__ void __launch_bounds__(KIN_THREADS, 2)
hpsi_kinetic_kernel(const __grid_constant__ CUtensorMap tmap, const DeviceTables<R> t, const KineticPlan<R> kp,
                    cplx<R> *__restrict__ out, cplx<R> *__restrict__ w1, cplx<R> *__restrict__ w2, R a2)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // staged boxes start on a KIN_STAGE_ALIGN boundary (the launch adds the slack)
    unsigned char *smem = smem_raw + ((KIN_STAGE_ALIGN - (smem_u32(smem_raw) & (KIN_STAGE_ALIGN - 1))) & (KIN_STAGE_ALIGN - 1));
    cplx<R> *BR = reinterpret_cast<cplx<R> *>(smem + 2 * (size_t)kp.stage_bytes);      // bridge-row partials
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * (size_t)kp.stage_bytes + KIN_BRIDGE_BYTES);
    constexpr int ALIGN = 16 / (int)sizeof(cplx<R>);   // nodes per 16 bytes (TMA start alignment)
    const int n = kp.n, nc = kp.nc, pitch = kp.box_r;
    const size_t nn = (size_t)n * n;
    const long long items = (long long)kp.ntr * kp.nct * nc;
    const long long per = (items + gridDim.x - 1) / gridDim.x;
    const long long first = (long long)blockIdx.x * per;
    const long long last = first + per < items ? first + per : items;
    if (first >= last) return;
    const unsigned box_bytes = (unsigned)((size_t)pitch * kp.box_c * sizeof(cplx<R>));

    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        mbar_fence_init();
    }
    __syncthreads();
    auto issue = [&](long long it, int stage) {
        const long long tile = it / nc;
        const int c = (int)(it % nc), tr = (int)(tile / kp.nct), tc = (int)(tile % kp.nct);
        const int x0 = kp.krbase[tr] / ALIGN * ALIGN;
        mbar_expect_tx(bar + stage, box_bytes);
        tma_load_3d(smem + (size_t)stage * kp.stage_bytes, &tmap, 2 * x0, kp.kcbase[tc], c, bar + stage);
    };
    if (threadIdx.x == 0) issue(first, 0);

    const int slot = threadIdx.x / KIN_ROWS, lane_row = threadIdx.x % KIN_ROWS;
    for (long long it = first; it < last; ++it) {
        const int k = (int)(it - first), stage = k & 1;
        const bool ok = mbar_wait_bounded(bar + stage, (unsigned)((k >> 1) & 1));
        if (__syncthreads_or(!ok)) {
            // a stage that never arrived: record it, wait (bounded) for the copy in flight, leave
            if (threadIdx.x == 0) {
                atomicExch(kp.err, 1);
                mbar_wait_bounded(bar + stage, (unsigned)((k >> 1) & 1));
            }
            return;
        }
        if (threadIdx.x == 0 && it + 1 < last) issue(it + 1, stage ^ 1);

        const long long tile = it / nc;
        const int c = (int)(it % nc), tr = (int)(tile / kp.nct), tc = (int)(tile % kp.nct);
        const int ea = kp.krow[tr], eb = kp.krow[tr + 1];
        const int r0 = kp.estart[ea], r1 = eb < kp.ne ? kp.estart[eb] : n;
        const cplx<R> *S = reinterpret_cast<const cplx<R> *>(smem + (size_t)stage * kp.stage_bytes);
        const int x0 = kp.krbase[tr] / ALIGN * ALIGN, y0 = kp.kcbase[tc];
        const int *slots = kp.kslot + tc * KIN_SLOTS * 3;
        const int c0 = kp.estart[slots[0]] + slots[1];   // first owned column of the tile

        // bridge-row partials: for every bridge row s_e (e >= max(ea, 1)) of the row tile and
        // every owned column, the previous element's last row applied along r1
        const int e_br = ea > 0 ? ea : 1, nbr = eb - e_br;
        const int ncol = slots[2] + slots[5] + slots[8] + slots[11];
        for (int idx = threadIdx.x; idx < nbr * ncol; idx += KIN_THREADS) {
            const int kb = idx / ncol, jj = idx - kb * ncol;
            const int e = e_br + kb, ep = e - 1, sp = kp.estart[ep], mp = kp.estart[e] - sp + 1;
            const int mpp = mp + (mp & 1), kf = kp.koff[ep];
            const cplx<R> *src = S + (c0 + jj - y0) * pitch + (sp - x0);
            const bool rp = kp.ereal[ep];
            cplx<R> s = mk<R>(0, 0);
            for (int b = 0; b < mp - 1; ++b) {
                const int kk = kf + b * mpp + (mp - 1);
                s = rp ? rfma<R>(__ldg(kp.tre + kk), src[b], s) : cfma<R>(mk<R>(__ldg(kp.tre + kk), __ldg(kp.tim + kk)), src[b], s);
            }
            BR[kb * KIN_BRCOLS + jj] = s;
        }
        __syncthreads();

        const int i = r0 + lane_row;
        const int f = slots[3 * slot], a0 = slots[3 * slot + 1], na = slots[3 * slot + 2];
        if (i >= r1 || na == 0) continue;
        const int il = i - x0, cq0 = kp.estart[f] + a0;
        cplx<R> acc[KIN_NA];
        if (VEL) {
#pragma unroll
            for (int q = 0; q < KIN_NA; ++q) acc[q] = mk<R>(0, 0);
            along_r2<R>(kp, kp.bre, kp.bim, S, pitch, il, y0, f, a0, na, acc);
#pragma unroll
            for (int q = 0; q < KIN_NA; ++q)
                if (q < na) w2[(size_t)i + (size_t)n * (cq0 + q) + nn * c] = acc[q];
#pragma unroll
            for (int q = 0; q < KIN_NA; ++q) acc[q] = mk<R>(0, 0);
            along_r1<R>(kp, kp.bre, kp.bim, S, pitch, i, x0, cq0, y0, na, true, acc);
#pragma unroll
            for (int q = 0; q < KIN_NA; ++q)
                if (q < na) w1[(size_t)i + (size_t)n * (cq0 + q) + nn * c] = acc[q];
        }
#pragma unroll
        for (int q = 0; q < KIN_NA; ++q) acc[q] = mk<R>(0, 0);
        along_r2<R>(kp, kp.tre, kp.tim, S, pitch, il, y0, f, a0, na, acc);
        along_r1<R>(kp, kp.tre, kp.tim, S, pitch, i, x0, cq0, y0, na, false, acc);
        const int e = kp.nodeelem[i];
        if (i == kp.estart[e] && e > 0) {   // bridge row: add its partials
            const cplx<R> *br = BR + (e - e_br) * KIN_BRCOLS + (cq0 - c0);
#pragma unroll
            for (int q = 0; q < KIN_NA; ++q)
                if (q < na) acc[q] = cadd<R>(acc[q], br[q]);
        }
#pragma unroll
        for (int q = 0; q < KIN_NA; ++q) {
            if (q < na) {
                const int j = cq0 + q;
                const cplx<R> x = S[(j - y0) * pitch + il];
                const size_t p = (size_t)i + (size_t)n * j + nn * c;
                const cplx<R> d = SEP ? cadd<R>(ldg<R>(t.d1 + i + (size_t)n * c), ldg<R>(t.d2 + j + (size_t)n * c))
                                      : ldg<R>(t.diag + p);
                cplx<R> v = cfma<R>(d, x, acc[q]);
                if (VEL) v = rfma<R>(a2, x, v);
                out[p] = v;
            }
        }
    }
}

// ---------------------------------------------------------------------------------
// Banded kinetic kernel on the FP64 tensor cores (complex128).
//
// Output fragments C[j][i] (8 columns j x 8 rows i of one channel) collect both electrons:
//   electron 1:  C[j][i] += sum_r S[r][j] T[i][r]     A = S^T (shared), B = row-group fragments
//   electron 2:  C[j][i] += sum_r T[j][r] S[i][r]     A = column-group fragments, B = S (shared)
// over the 4-node k-steps of each group's window; complex products take two (real T) or
// four (complex T) mma.sync m8n8k4 f64 per k-step.  A CTA of 8 warps owns a 64 x 32
// tile: warp w keeps the fragments of row group w in registers and all four column
// groups' fragments come from shared memory (staged when the column tile changes).
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// acc += A B for complex operands; B_real / A_real select the two-product form.
__device__ __forceinline__ void cmma_ab(double (&cr)[2], double (&ci)[2], double2 a, double2 b, bool b_real)
{
    dmma(cr[0], cr[1], a.x, b.x);
    dmma(ci[0], ci[1], a.y, b.x);
    if (!b_real) {
        dmma(cr[0], cr[1], -a.y, b.y);
        dmma(ci[0], ci[1], a.x, b.y);
    }
}

__device__ __forceinline__ void cmma_ba(double (&cr)[2], double (&ci)[2], double2 a, double2 b, bool a_real)
{
    dmma(cr[0], cr[1], a.x, b.x);
    dmma(ci[0], ci[1], a.x, b.y);
    if (!a_real) {
        dmma(cr[0], cr[1], -a.y, b.y);
        dmma(ci[0], ci[1], a.y, b.x);
    }
}

// S element as complex FP64 (complex64 storage is widened exactly)
__device__ __forceinline__ double2 s_load(const double2 *p) { return *p; }
__device__ __forceinline__ double2 s_load(const float2 *p)
{
    const float2 v = *p;
    return make_double2((double)v.x, (double)v.y);
}

// Electron 1 over the window of this warp's row group: block q covers columns j0 + (0..7).
template <typename C>
__device__ __forceinline__ void band_r1(const C *S, int P, int x0, int y0, int j0, int glo, int gks, bool real,
                                        const double2 (&rf)[BAND_KS], int lr, int lk, double (&cr)[2], double (&ci)[2])
{
    const C *a = S + (j0 + lr - y0) * P + (glo + lk - x0);
#pragma unroll
    for (int s = 0; s < BAND_KS; ++s)
        if (s < gks) cmma_ab(cr, ci, s_load(a + 4 * s), rf[s], real);
}

// Electron 2 over the window of column group gc, fragments `cf` (k-step major, 32 lanes).
template <typename C>
__device__ __forceinline__ void band_r2(const C *S, int P, int x0, int y0, int i0, int glo, int gks, bool real,
                                        const double2 *cf, int lane, int lr, int lk, double (&cr)[2], double (&ci)[2])
{
    const C *b = S + (glo + lk - y0) * P + (i0 + lr - x0);
#pragma unroll
    for (int s = 0; s < BAND_KS; ++s)
        if (s < gks) cmma_ba(cr, ci, cf[s * 32 + lane], s_load(b + 4 * s * P), real);
}

// The same two sweeps for all BAND_CG column groups of the tile at once: the k-step loop
// is outermost, so every k-step issues 2 * BAND_CG independent accumulation chains (the
// DMMA latency of one chain is hidden behind the others).  Column group q covers columns
// j0 + 8 q + (0..7); groups past the grid have gks_c[q] = 0 (and zero fragments).
template <typename C>
__device__ __forceinline__ void band_r1_tile(const C *S, int P, int x0, int y0, int j0, int glo, int gks, bool real,
                                             const double2 (&rf)[BAND_KS], int lr, int lk,
                                             double (&cr)[BAND_CG][2], double (&ci)[BAND_CG][2])
{
    const C *a = S + (j0 + lr - y0) * P + (glo + lk - x0);
#pragma unroll
    for (int s = 0; s < BAND_KS; ++s)
        if (s < gks) {
#pragma unroll
            for (int q = 0; q < BAND_CG; ++q) cmma_ab(cr[q], ci[q], s_load(a + 8 * q * P + 4 * s), rf[s], real);
        }
}

template <typename C>
__device__ __forceinline__ void band_r2_tile(const C *S, int P, int x0, int y0, int i0, const int (&glo_c)[BAND_CG],
                                             const int (&gks_c)[BAND_CG], const bool (&real_c)[BAND_CG],
                                             const double2 *cf, size_t cf_stride, int lane, int lr, int lk,
                                             double (&cr)[BAND_CG][2], double (&ci)[BAND_CG][2])
{
#pragma unroll
    for (int s = 0; s < BAND_KS; ++s)
#pragma unroll
        for (int q = 0; q < BAND_CG; ++q)
            if (s < gks_c[q])
                cmma_ba(cr[q], ci[q], cf[q * cf_stride + s * 32 + lane],
                        s_load(S + (glo_c[q] + lk + 4 * s - y0) * P + (i0 + lr - x0)), real_c[q]);
}

template <typename R> __device__ __forceinline__ cplx<R> narrow(double re, double im) { return mk<R>((R)re, (R)im); }

// Work items are (row tile, column tile, channel of the batch): the batch's instances are
// consecutive blocks of nc channels, so instance b owns channels [b nc, (b + 1) nc) of the
// 3-D TMA map and of every array.
// NST = 2: two TMA stages (the next item's box lands while this one is computed), one CTA
// per SM; NST = 1: one stage, the next box is requested after the item, and the register
// budget admits two CTAs per SM, which hide each other's waits.
template <typename R, bool VEL, bool SEP, int NST>
__global__ void __launch_bounds__(BAND_THREADS, NST == 1 ? 2 : 1)
hpsi_band_kernel(const __grid_constant__ CUtensorMap tmap, const DeviceTables<R> t, const BandPlan<R> bp,
                 cplx<R> *__restrict__ out, cplx<R> *__restrict__ w1, cplx<R> *__restrict__ w2,
                 const __grid_constant__ FieldBatch fb)
{
    typedef cplx<R> C;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *smem = smem_raw + ((KIN_STAGE_ALIGN - (smem_u32(smem_raw) & (KIN_STAGE_ALIGN - 1))) & (KIN_STAGE_ALIGN - 1));
    double2 *CF = reinterpret_cast<double2 *>(smem + NST * (size_t)bp.stage_bytes);   // [BAND_CG][BAND_KS][32]
    double2 *CFB = CF + BAND_CG * BAND_KS * 32;   // velocity gauge: the B fragments of the same groups
    uint64_t *bar = reinterpret_cast<uint64_t *>(CFB + (VEL ? BAND_CG * BAND_KS * 32 : 0));
    constexpr int ALIGN = 16 / (int)sizeof(C);   // nodes per 16 bytes (TMA start alignment)
    if (fb.skip && *fb.skip) return;   // the solve that enqueued this apply has converged
    const int n = bp.n, nc = bp.nc, P = bp.box_r, G = bp.ngroup, nch = nc * fb.count;
    const size_t nn = (size_t)n * n;
    const long long items = (long long)bp.ntr * bp.nct * nch;
    const long long per = (items + gridDim.x - 1) / gridDim.x;
    const long long first = (long long)blockIdx.x * per;
    const long long last = first + per < items ? first + per : items;
    if (first >= last) return;
    const unsigned box_bytes = (unsigned)((size_t)P * bp.box_c * sizeof(C));

    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        mbar_fence_init();
    }
    __syncthreads();
    auto issue = [&](long long it, int stage) {
        const long long tile = it / nch;
        const int c = (int)(it % nch), tr = (int)(tile / bp.nct), tc = (int)(tile % bp.nct);
        mbar_expect_tx(bar + stage, box_bytes);
        tma_load_3d(smem + (size_t)stage * bp.stage_bytes, &tmap, 2 * (bp.brbase[tr] / ALIGN * ALIGN), bp.bcbase[tc], c,
                    bar + stage);
    };
    if (threadIdx.x == 0) issue(first, 0);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, lr = lane >> 2, lk = lane & 3;
    int cur_tr = -1, cur_tc = -1;
    double2 rf[BAND_KS];
    int glo_r = 0, gks_r = 0;
    bool real_r = true;
    for (long long it = first; it < last; ++it) {
        const int k = (int)(it - first), stage = NST == 2 ? (k & 1) : 0;
        const unsigned parity = NST == 2 ? (unsigned)((k >> 1) & 1) : (unsigned)(k & 1);
        const bool ok = mbar_wait_bounded(bar + stage, parity);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicExch(bp.err, 1);
                mbar_wait_bounded(bar + stage, parity);
            }
            return;
        }
        if (NST == 2 && threadIdx.x == 0 && it + 1 < last) issue(it + 1, stage ^ 1);
        const long long tile = it / nch;
        const int c = (int)(it % nch), tr = (int)(tile / bp.nct), tc = (int)(tile % bp.nct);
        const int cc = c % nc, inst = c / nc;   // channel within its instance, instance
        if (tc != cur_tc) {   // CTA-uniform: stage the column groups' fragments
            for (int idx = threadIdx.x; idx < BAND_CG * BAND_KS * 32; idx += BAND_THREADS) {
                const int g = tc * BAND_CG + idx / (BAND_KS * 32);
                CF[idx] = g < G ? bp.frag[(size_t)g * BAND_KS * 32 + idx % (BAND_KS * 32)] : make_double2(0, 0);
                if (VEL)
                    CFB[idx] = g < G ? bp.fragb[(size_t)g * BAND_KS * 32 + idx % (BAND_KS * 32)] : make_double2(0, 0);
            }
            cur_tc = tc;
            __syncthreads();
        }
        const int gr = tr * BAND_WARPS + warp;
        if (tr != cur_tr) {   // this warp's row-group fragments
            cur_tr = tr;
            if (gr < G) {
#pragma unroll
                for (int s = 0; s < BAND_KS; ++s) rf[s] = bp.frag[((size_t)gr * BAND_KS + s) * 32 + lane];
                glo_r = bp.glo[gr]; gks_r = bp.gks[gr]; real_r = bp.greal[gr] & 1;
            }
        }
        if (gr < G) {   // warps past the last row group only keep the CTA's barriers
        const C *S = reinterpret_cast<const C *>(smem + (size_t)stage * bp.stage_bytes);
        const int x0 = bp.brbase[tr] / ALIGN * ALIGN, y0 = bp.bcbase[tc], i0 = gr * BAND_G;
        int glo_c[BAND_CG], gks_c[BAND_CG];
        bool real_c[BAND_CG], breal_c[BAND_CG];
#pragma unroll
        for (int q = 0; q < BAND_CG; ++q) {
            const int gc = tc * BAND_CG + q;
            const bool in = gc < G;
            glo_c[q] = in ? bp.glo[gc] : 0;
            gks_c[q] = in ? bp.gks[gc] : 0;
            real_c[q] = in ? (bp.greal[gc] & 1) != 0 : true;
            breal_c[q] = in ? (bp.greal[gc] & 2) != 0 : true;
        }
        const int j0 = tc * BAND_TC;
        if (VEL) {   // commutator stencils W1 (electron 1), W2 (electron 2) with the B fragments
            double2 bf[BAND_KS];
#pragma unroll
            for (int s = 0; s < BAND_KS; ++s) bf[s] = bp.fragb[((size_t)gr * BAND_KS + s) * 32 + lane];
            const bool breal_r = (bp.greal[gr] & 2) != 0;
            double cr[BAND_CG][2] = {}, ci[BAND_CG][2] = {};
            band_r1_tile(S, P, x0, y0, j0, glo_r, gks_r, breal_r, bf, lr, lk, cr, ci);
            double dr[BAND_CG][2] = {}, di[BAND_CG][2] = {};
            band_r2_tile(S, P, x0, y0, i0, glo_c, gks_c, breal_c, CFB, (size_t)BAND_KS * 32, lane, lr, lk, dr, di);
#pragma unroll
            for (int q = 0; q < BAND_CG; ++q)
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int i = i0 + 2 * lk + u, j = j0 + 8 * q + lr;
                    if (i < n && j < n) {
                        w1[(size_t)i + (size_t)n * j + nn * c] = narrow<R>(cr[q][u], ci[q][u]);
                        w2[(size_t)i + (size_t)n * j + nn * c] = narrow<R>(dr[q][u], di[q][u]);
                    }
                }
        }
        const double *fv = fb.f[inst];
        const double a2 = VEL ? fv[0] * fv[0] + fv[1] * fv[1] + fv[2] * fv[2] : 0.0;
        double cr[BAND_CG][2] = {}, ci[BAND_CG][2] = {};
        band_r1_tile(S, P, x0, y0, j0, glo_r, gks_r, real_r, rf, lr, lk, cr, ci);
        band_r2_tile(S, P, x0, y0, i0, glo_c, gks_c, real_c, CF, (size_t)BAND_KS * 32, lane, lr, lk, cr, ci);
#pragma unroll
        for (int q = 0; q < BAND_CG; ++q)
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int i = i0 + 2 * lk + u, j = j0 + 8 * q + lr;
                if (i < n && j < n) {
                    const double2 x = s_load(S + (j - y0) * P + (i - x0));
                    const size_t p = (size_t)i + (size_t)n * j;
                    const C dd = SEP ? cadd<R>(ldg<R>(t.d1 + i + (size_t)n * cc), ldg<R>(t.d2 + j + (size_t)n * cc))
                                     : ldg<R>(t.diag + p + nn * cc);
                    double2 v = cfma<double>(make_double2((double)dd.x, (double)dd.y), x, make_double2(cr[q][u], ci[q][u]));
                    if (VEL) v = rfma<double>(a2, x, v);
                    out[p + nn * c] = narrow<R>(v.x, v.y);
                }
            }
        }
        if (NST == 1) {   // every warp is done with the stage: request the next box into it
            __syncthreads();
            if (threadIdx.x == 0 && it + 1 < last) issue(it + 1, 0);
        }
    }
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

}  // namespace

// Multiprocessor count of a device (cached; 148 on B200 when the query fails).
int sm_count(int device)
{
    static int counts[64] = {0};
    if (device < 0 || device >= 64) return 148;
    if (!counts[device]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0) v = 148;
        counts[device] = v;
    }
    return counts[device];
}

// CTAs of one kernel that fit on an SM at a block size and dynamic shared memory (occupancy
// calculator, cached per kernel and size; at least 1).
int resident_ctas(const void *kernel, int threads, size_t smem)
{
    struct Entry { const void *k; int threads; size_t smem; int device; int n; };
    static thread_local Entry cache[16];
    static thread_local int next = 0;
    int device = 0;
    cudaGetDevice(&device);
    for (const Entry &e : cache)
        if (e.k == kernel && e.threads == threads && e.smem == smem && e.device == device) return e.n;
    int n = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess || n < 1) n = 1;
    cache[next] = {kernel, threads, smem, device, n};
    next = (next + 1) % 16;
    return n;
}

// TMA map of psi(re/im, r1, r2 channel) over nc channels (every instance of a batch) with a
// (2 box_r, box_c, 1) box, keyed by (buffer, kind) in the
// operator's cache of recently used buffers (a Krylov basis reuses the same few), else
// encoded now; `kind` encodes the kernel family, precision and batch size.  Returns null
// when encoding fails.
const CUtensorMap *psi_map(he_operator *h, int kind, const void *psi, int n, int nc, int box_r, int box_c,
                           size_t real_bytes)
{
    for (auto &e : h->tmaps)
        if (e.base == psi && e.kind == kind) return &e.map;
    auto &e = h->tmaps[h->tmap_next];
    h->tmap_next = (h->tmap_next + 1) % (int)(sizeof(h->tmaps) / sizeof(h->tmaps[0]));
    const cuuint64_t dims[3] = {2 * (cuuint64_t)n, (cuuint64_t)n, (cuuint64_t)nc};
    const cuuint64_t strides[2] = {2 * (cuuint64_t)n * real_bytes, 2 * (cuuint64_t)n * n * real_bytes};
    const cuuint32_t box[3] = {2 * (cuuint32_t)box_r, (cuuint32_t)box_c, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    e.base = nullptr;
    const CUresult r = tensor_map_encoder()(&e.map, real_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                            3, const_cast<void *>(psi), dims, strides, box, es,
                                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return nullptr;
    e.base = psi;
    e.kind = kind;
    return &e.map;
}

// True when the kinetic kernel can stage `psi` with TMA: 16-byte aligned base and rows
// (the r1 extent in bytes) a multiple of 16 bytes.
template <typename R> bool kinetic_usable(const KineticPlan<R> &kp, const void *psi)
{
    return kp.ntr > 0 && (reinterpret_cast<uintptr_t>(psi) & 15) == 0 && ((size_t)kp.n * sizeof(cplx<R>)) % 16 == 0 &&
           tensor_map_encoder() != nullptr;
}

template <typename R>
int launch_kinetic(he_operator *h, const DeviceTables<R> &t, const KineticPlan<R> &kp, const cplx<R> *psi,
                   cplx<R> *out, cplx<R> *w1, cplx<R> *w2, R a2, int velocity, cudaStream_t stream)
{
    const CUtensorMap *mp = psi_map(h, sizeof(R) == 8 ? 1 : 2, psi, kp.n, kp.nc, kp.box_r, kp.box_c, sizeof(R));
    if (!mp) return he_fail(HE_ERR_CUDA, "cuTensorMapEncodeTiled failed", __FILE__, __LINE__);
    const CUtensorMap map = *mp;
    const size_t smem = 2 * (size_t)kp.stage_bytes + KIN_BRIDGE_BYTES + 16 + KIN_STAGE_ALIGN;
    const long long items = (long long)kp.ntr * kp.nct * kp.nc;
    const unsigned grid = (unsigned)std::min<long long>(items, 2LL * sm_count(h->device));
#define HE_KINETIC(V, S)                                                                                   \
    do {                                                                                                   \
        auto kern = hpsi_kinetic_kernel<R, V, S>;                                                          \
        HE_CUDA_TRY(he_smem_limit(reinterpret_cast<const void *>(kern), smem));   \
        kern<<<grid, KIN_THREADS, smem, stream>>>(map, t, kp, out, w1, w2, a2);                            \
    } while (0)
    if (velocity) { if (t.diag_separable) HE_KINETIC(true, true); else HE_KINETIC(true, false); }
    else { if (t.diag_separable) HE_KINETIC(false, true); else HE_KINETIC(false, false); }
#undef HE_KINETIC
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

// True when the banded kernel can stage `psi` with TMA: 16-byte aligned base and rows
// (the r1 extent in bytes) a multiple of 16 bytes.
template <typename R> bool band_usable(const BandPlan<R> &bp, const void *psi)
{
    return bp.ntr > 0 && (reinterpret_cast<uintptr_t>(psi) & 15) == 0 && ((size_t)bp.n * sizeof(cplx<R>)) % 16 == 0 &&
           tensor_map_encoder() != nullptr;
}

template <typename R>
int launch_band(he_operator *h, const DeviceTables<R> &t, const BandPlan<R> &bp, const cplx<R> *psi, cplx<R> *out,
                cplx<R> *w1, cplx<R> *w2, const FieldBatch &fb, int velocity, cudaStream_t stream)
{
    const CUtensorMap *mp = psi_map(h, (sizeof(R) == 8 ? 0 : 3) + 8 * fb.count, psi, bp.n, bp.nc * fb.count, bp.box_r,
                                    bp.box_c, sizeof(R));
    if (!mp) return he_fail(HE_ERR_CUDA, "cuTensorMapEncodeTiled failed", __FILE__, __LINE__);
    const CUtensorMap map = *mp;
    // length gauge: the single-stage form at two CTAs per SM when the operator asks for it
    // (he_set_band_stages); the velocity gauge needs the registers of one CTA per SM
    const int nst = (!velocity && h->band_stages[sizeof(R) == 8 ? 0 : 1] == 1) ? 1 : 2;
    const size_t smem = nst * (size_t)bp.stage_bytes +
                        (velocity ? 2 : 1) * (size_t)BAND_CG * BAND_KS * 32 * sizeof(double2) + 16 + KIN_STAGE_ALIGN;
    const long long items = (long long)bp.ntr * bp.nct * bp.nc * fb.count;
#define HE_BAND(V, S, N)                                                                                   \
    do {                                                                                                   \
        auto kern = hpsi_band_kernel<R, V, S, N>;                                                          \
        HE_CUDA_TRY(he_smem_limit(reinterpret_cast<const void *>(kern), smem));                            \
        const int per_sm = resident_ctas(reinterpret_cast<const void *>(kern), BAND_THREADS, smem);        \
        const unsigned grid = (unsigned)std::min<long long>(items, (long long)per_sm * sm_count(h->device)); \
        kern<<<grid, BAND_THREADS, smem, stream>>>(map, t, bp, out, w1, w2, fb);                           \
    } while (0)
    if (velocity) { if (t.diag_separable) HE_BAND(true, true, 2); else HE_BAND(true, false, 2); }
    else if (nst == 1) { if (t.diag_separable) HE_BAND(false, true, 1); else HE_BAND(false, false, 1); }
    else { if (t.diag_separable) HE_BAND(false, true, 2); else HE_BAND(false, false, 2); }
#undef HE_BAND
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

template bool band_usable<double>(const BandPlan<double> &, const void *);
template bool band_usable<float>(const BandPlan<float> &, const void *);
template int launch_band<double>(he_operator *, const DeviceTables<double> &, const BandPlan<double> &, const double2 *,
                                 double2 *, double2 *, double2 *, const FieldBatch &, int, cudaStream_t);
template int launch_band<float>(he_operator *, const DeviceTables<float> &, const BandPlan<float> &, const float2 *,
                                float2 *, float2 *, float2 *, const FieldBatch &, int, cudaStream_t);
template bool kinetic_usable<double>(const KineticPlan<double> &, const void *);
template bool kinetic_usable<float>(const KineticPlan<float> &, const void *);
template int launch_kinetic<double>(he_operator *, const DeviceTables<double> &, const KineticPlan<double> &,
                                    const double2 *, double2 *, double2 *, double2 *, double, int, cudaStream_t);
template int launch_kinetic<float>(he_operator *, const DeviceTables<float> &, const KineticPlan<float> &,
                                   const float2 *, float2 *, float2 *, float2 *, float, int, cudaStream_t);

}  // namespace he
