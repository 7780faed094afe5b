// Separable ionic resolvent preconditioner (python/implicit.py:13-39) on the device.
//
// For channel c with one-electron angular momenta (l1, l2) and the eigendecompositions
// H_l = S_l diag(e_l) S_l^-1 of the ionic radial Hamiltonians (computed on the host):
//   Z_c = S_{l1}^-1 Psi_c (S_{l2}^-1)^T,   Z_c(i,j) /= 1 + i alpha (e_{l1}(i) + e_{l2}(j) + shift),
//   Y_c = S_{l1} Z_c S_{l2}^T
// with Psi_c the n x n column-major slice psi(:, :, c) (the reference's u[c] is its
// transpose, so I2 u I1^T there is I1 Psi I2^T here).
//
// Every two-sided product A X B^T is two launches of one kernel shape, a left product
// with a transposed store: out_c = (M_{sel(c)} X_c)^T.  Applied with M = A and then with
// M = B it gives (B (A X)^T)^T = A X B^T, and the transposed store keeps every operand
// K-contiguous.  The resolvent division is fused into the store of the second product.
//
// complex128: FP64 tensor cores, mma.sync.m8n8k4.f64 (four real MMAs per complex
//   product), cp.async-staged output tiles (32 x 32 per warp) in four shared-memory stages.
// complex64 (the reference's precision='complex64'): the fifth-generation tensor cores,
//   tcgen05.mma kind::tf32 with TMEM accumulators and TMA-loaded, 128-byte-swizzled
//   operands.  The complex product is the real GEMM of its real embedding,
//   [Re; Im](M X) = [[Re M, -Im M], [Im M, Re M]] [Re X; Im X], K-major on both sides
//   because psi stores (Re, Im) interleaved along the contraction index.  Each operand is
//   split into two TF32 parts, x = hi + lo, and D = Ah Xh + Ah Xl + Al Xh accumulates in
//   FP32 (three MMAs per K slice), which keeps the product at FP32-class accuracy
//   (relative error about 2^-21) for the flexible GMRES that consumes it.  The real
//   embeddings of S and S^-1 and their TF32 parts are built once at creation.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "operator.cuh"
#include "sm100.cuh"

namespace he {

// ---------------------------------------------------------------------------------------
// complex128: DMMA GEMM
// ---------------------------------------------------------------------------------------
// Tile of one CTA: WM x WN warps of 32 x 32 complex outputs each, DG_BK = 8 contraction
// steps per stage, DG_STAGES cp.async stages; shared rows padded to DG_LD complex values so
// that the fragment loads (16-byte complex values, 8 rows x 4 columns per quarter warp) hit
// distinct banks.  Two shapes: 64 x 128 (2 x 4 warps) for large n, 32 x 64 (1 x 2 warps)
// when the large tiles would not give every SM two CTAs.
constexpr int DG_BK = 8;
constexpr int DG_LD = DG_BK + 4;
constexpr int DG_STAGES = 4;
template <int WM, int WN, int FM, int FN> constexpr size_t dg_smem()
{
    return (size_t)DG_STAGES * (8 * FM * WM + 8 * FN * WN) * DG_LD * sizeof(double2);
}

// Resolvent division fused into a product's store: out /= 1 + i alpha (e_row + e_col + shift),
// e_row = evals[lrow[c]][row], e_col = evals[lcol[c]][col].
template <typename R> struct Resolvent {
    const cplx<R> *evals;                        // nl x n
    const int *lrow, *lcol;                      // per channel
    cplx<R> alpha;
    R shift;
    int on;
};

template <typename R>
__device__ __forceinline__ cplx<R> resolve(const Resolvent<R> &rs, int n, int c, int row, int col, cplx<R> v)
{
    const cplx<R> e1 = rs.evals[(size_t)rs.lrow[c] * n + row], e2 = rs.evals[(size_t)rs.lcol[c] * n + col];
    const cplx<R> es = mk<R>(e1.x + e2.x + rs.shift, e1.y + e2.y);
    const cplx<R> ia = mk<R>(-rs.alpha.y, rs.alpha.x);
    const cplx<R> den = cfma<R>(ia, es, mk<R>(1, 0));
    const R d2 = cabs2<R>(den);
    return mk<R>((v.x * den.x + v.y * den.y) / d2, (v.y * den.x - v.x * den.y) / d2);
}

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(c0), "+d"(c1) : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp16(void *smem, const void *gmem, bool ok)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(ok ? 16 : 0) : "memory");
}

// out_c = (M_{sel[c]} X_c)^T for every channel c (grid.z): M row-major n x n (mats + l n^2),
// X_c(k, j) = x[(c n + j) n + k], out_c(j, i) = out[(c n + i) n + j].
template <int WM, int WN, int FM, int FN>
__global__ void __launch_bounds__(32 * WM * WN, 1)
sep_dgemm_kernel(int n, const double2 *__restrict__ mats, const int *__restrict__ sel, const double2 *__restrict__ x,
                 double2 *__restrict__ out, Resolvent<double> rs, const int *gate)
{
    if (gate && *gate) return;
    constexpr int BM = 8 * FM * WM, BN = 8 * FN * WN, THREADS = 32 * WM * WN;
    constexpr int A_ELEMS = BM * DG_LD, B_ELEMS = BN * DG_LD;
    extern __shared__ double2 dsm[];
    double2 *As = dsm, *Bs = dsm + DG_STAGES * A_ELEMS;
    const int c = blockIdx.z, i0 = blockIdx.x * BM, j0 = blockIdx.y * BN;
    const size_t nn = (size_t)n * n;
    const double2 *M = mats + (size_t)sel[c] * nn;
    const double2 *X = x + (size_t)c * nn;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int wm = (warp % WM) * 8 * FM, wn = (warp / WM) * 8 * FN;
    const int nk = (n + DG_BK - 1) / DG_BK;

    auto load = [&](int kt, int stage) {
        const int k0 = kt * DG_BK;
        double2 *a = As + stage * A_ELEMS, *b = Bs + stage * B_ELEMS;
        for (int e = tid; e < BM * DG_BK; e += THREADS) {
            const int r = e / DG_BK, k = e % DG_BK, gi = i0 + r, gk = k0 + k;
            const bool ok = gi < n && gk < n;
            cp16(a + r * DG_LD + k, ok ? M + (size_t)gi * n + gk : M, ok);
        }
        for (int e = tid; e < BN * DG_BK; e += THREADS) {
            const int r = e / DG_BK, k = e % DG_BK, gj = j0 + r, gk = k0 + k;
            const bool ok = gj < n && gk < n;
            cp16(b + r * DG_LD + k, ok ? X + (size_t)gj * n + gk : X, ok);
        }
    };

    double cr[FM][FN][2], ci[FM][FN][2];
#pragma unroll
    for (int a = 0; a < FM; ++a)
#pragma unroll
        for (int b = 0; b < FN; ++b) cr[a][b][0] = cr[a][b][1] = ci[a][b][0] = ci[a][b][1] = 0.0;

#pragma unroll
    for (int s = 0; s < DG_STAGES - 1; ++s) {
        if (s < nk) load(s, s);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int kt = 0; kt < nk; ++kt) {
        asm volatile("cp.async.wait_group %0;" ::"n"(DG_STAGES - 2) : "memory");
        __syncthreads();
        if (kt + DG_STAGES - 1 < nk) load(kt + DG_STAGES - 1, (kt + DG_STAGES - 1) % DG_STAGES);
        asm volatile("cp.async.commit_group;" ::: "memory");
        const double2 *a = As + (kt % DG_STAGES) * A_ELEMS, *b = Bs + (kt % DG_STAGES) * B_ELEMS;
#pragma unroll
        for (int kk = 0; kk < DG_BK; kk += 4) {
            double2 fa[FM], fb[FN];
#pragma unroll
            for (int m = 0; m < FM; ++m) fa[m] = a[(wm + m * 8 + (lane >> 2)) * DG_LD + kk + (lane & 3)];
#pragma unroll
            for (int q = 0; q < FN; ++q) fb[q] = b[(wn + q * 8 + (lane >> 2)) * DG_LD + kk + (lane & 3)];
            // the two halves of each complex product go 2 FM FN MMAs apart, so no MMA waits
            // on the one before it
#pragma unroll
            for (int m = 0; m < FM; ++m)
#pragma unroll
                for (int q = 0; q < FN; ++q) {
                    dmma(cr[m][q][0], cr[m][q][1], fa[m].x, fb[q].x);
                    dmma(ci[m][q][0], ci[m][q][1], fa[m].x, fb[q].y);
                }
#pragma unroll
            for (int m = 0; m < FM; ++m) {
                const double nai = -fa[m].y;
#pragma unroll
                for (int q = 0; q < FN; ++q) {
                    dmma(cr[m][q][0], cr[m][q][1], nai, fb[q].y);
                    dmma(ci[m][q][0], ci[m][q][1], fa[m].y, fb[q].x);
                }
            }
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");

    double2 *O = out + (size_t)c * nn;
#pragma unroll
    for (int m = 0; m < FM; ++m) {
        const int i = i0 + wm + m * 8 + (lane >> 2);
        if (i >= n) continue;
#pragma unroll
        for (int q = 0; q < FN; ++q)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = j0 + wn + q * 8 + 2 * (lane & 3) + h;
                if (j >= n) continue;
                double2 v = make_double2(cr[m][q][h], ci[m][q][h]);
                if (rs.on) v = resolve<double>(rs, n, c, i, j, v);
                O[(size_t)i * n + j] = v;
            }
    }
}

// ---------------------------------------------------------------------------------------
// complex64: tcgen05 TF32 GEMM of the real embedding, split operands (3 products)
// ---------------------------------------------------------------------------------------
constexpr int TG_BM = 128;                       // output real rows (i, re/im) per CTA = TMEM lanes
constexpr int TG_BK = 32;                        // contraction floats per stage (one swizzle atom)
constexpr int TG_BN_MAX = 256;                   // output columns per CTA, at most (TMEM columns)
constexpr int TG_STAGES = 2;
constexpr int TG_THREADS = 128;                  // 4 warps: producer, MMA issuer, TMEM owner; all store
constexpr int TG_A_BYTES = TG_BM * TG_BK * 4;
constexpr int TG_B_BYTES = TG_BN_MAX * TG_BK * 4;
constexpr int TG_STAGE_BYTES = 2 * TG_A_BYTES + 2 * TG_B_BYTES;          // hi and lo of A and B
constexpr size_t TG_SMEM = (size_t)TG_STAGES * TG_STAGE_BYTES + 1024 + 256;

struct TcArgs {
    int n, nc, bn, kt, passes;
    int arows;                                   // rows of one matrix's embedding (2 n)
    const int *sel;
    int mode;                                    // 0: write TF32 hi/lo planes, 1: write complex128
    float *hi, *lo;                              // planes, row (c n + i), ld floats
    int ld;
    double2 *y;                                  // complex128 output, ((c n + i) n + j)
    Resolvent<float> rs;
    int *err;
    const int *gate;                             // non-zero at launch: return without work
};

__global__ void __launch_bounds__(TG_THREADS, 1)
sep_tf32_kernel(const __grid_constant__ CUtensorMap map_ah, const __grid_constant__ CUtensorMap map_al,
                const __grid_constant__ CUtensorMap map_xh, const __grid_constant__ CUtensorMap map_xl, TcArgs g)
{
    using namespace sm100;
    if (g.gate && *g.gate) return;               // uniform over the CTA, before any TMEM use
    extern __shared__ uint8_t tsm_raw[];
    const unsigned base_s = saddr(tsm_raw);
    uint8_t *tsm = tsm_raw + (((base_s + 1023u) & ~1023u) - base_s);  // 1024-byte aligned tiles
    uint64_t *full = reinterpret_cast<uint64_t *>(tsm + TG_STAGES * TG_STAGE_BYTES);
    uint64_t *empty = full + TG_STAGES;
    uint64_t *done = empty + TG_STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    __shared__ int lost;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * TG_BM, ntile = blockIdx.y, c = blockIdx.z;
    const int n = g.n, bn = g.bn, j0 = ntile * bn;
    const int mrow = g.sel[c] * g.arows + m0;    // first row of this tile in the stacked embeddings
    const int xrow = c * n + j0;                 // first operand row (output column) of this tile
    const bool split = g.passes == 3;

    if (threadIdx.x == 0) {
        lost = 0;
        for (int s = 0; s < TG_STAGES; ++s) { bar_init(&full[s], 1); bar_init(&empty[s], 1); }
        bar_init(done, 1);
        bar_fence_init();
        prefetch_map(&map_ah); prefetch_map(&map_xh);
        if (split) { prefetch_map(&map_al); prefetch_map(&map_xl); }
    }
    if (warp == 2) tmem_alloc(tmem_slot, TG_BN_MAX);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // producer: stage s holds [Ah | Al | Xh | Xl] of one K slice
        const unsigned bytes = (unsigned)(split ? 2 : 1) * (TG_A_BYTES + bn * TG_BK * 4);
        for (int kt = 0; kt < g.kt; ++kt) {
            const int s = kt % TG_STAGES;
            if (kt >= TG_STAGES && !bar_wait(&empty[s], ((kt / TG_STAGES) & 1) ^ 1)) { lost = 1; break; }
            uint8_t *st = tsm + s * TG_STAGE_BYTES;
            bar_expect_tx(&full[s], bytes);
            const int k0 = kt * TG_BK;
            tma_load_2d(st, &map_ah, k0, mrow, &full[s]);
            tma_load_2d(st + 2 * TG_A_BYTES, &map_xh, k0, xrow, &full[s]);
            if (split) {
                tma_load_2d(st + TG_A_BYTES, &map_al, k0, mrow, &full[s]);
                tma_load_2d(st + 2 * TG_A_BYTES + TG_B_BYTES, &map_xl, k0, xrow, &full[s]);
            }
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: 4 K slices of 8 per stage, 1 or 3 products each
        const uint32_t idesc = idesc_tf32(TG_BM, bn);
        for (int kt = 0; kt < g.kt; ++kt) {
            const int s = kt % TG_STAGES;
            if (!bar_wait(&full[s], (kt / TG_STAGES) & 1)) { lost = 1; break; }
            fence_after_sync();
            const unsigned st = saddr(tsm + s * TG_STAGE_BYTES);
#pragma unroll
            for (int k = 0; k < TG_BK / 8; ++k) {
                const unsigned off = (unsigned)k * 32u;
                const uint64_t ah = desc_k_sw128(st + off), xh = desc_k_sw128(st + 2 * TG_A_BYTES + off);
                mma_tf32(tmem, ah, xh, idesc, (kt | k) != 0);
                if (split) {
                    const uint64_t al = desc_k_sw128(st + TG_A_BYTES + off);
                    const uint64_t xl = desc_k_sw128(st + 2 * TG_A_BYTES + TG_B_BYTES + off);
                    mma_tf32(tmem, ah, xl, idesc, 1);
                    mma_tf32(tmem, al, xh, idesc, 1);
                }
            }
            mma_commit(&empty[s]);
        }
        mma_commit(done);
    }
    __syncwarp();

    // epilogue: lane m of TMEM = output real row m0 + m = (i, re/im); pairs of lanes swap
    // halves so that each thread stores 16 consecutive complex outputs of one row i.
    const bool ready = bar_wait(done, 0);
    fence_after_sync();
    if (!ready) lost = 1;
    const int row = m0 + warp * 32 + lane;
    const int i = row >> 1, part = row & 1;
    if (ready && !lost) {
        for (int col = 0; col < bn; col += 32) {
            float v[32];
            tmem_load32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col, v);
            float re[16], im[16];
#pragma unroll
            for (int t = 0; t < 16; ++t) {
                const float other = __shfl_xor_sync(0xffffffffu, part ? v[t] : v[t + 16], 1);
                re[t] = part ? other : v[t];
                im[t] = part ? v[t + 16] : other;
            }
            const int jb = j0 + col + 16 * part;      // first output column of this thread
            const int count = min(16, min(n, j0 + bn) - jb);   // inside the channel and this tile
            if (i >= n || count <= 0) continue;
            if (g.rs.on)
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    if (t < count) {
                        const float2 w = resolve<float>(g.rs, n, c, i, jb + t, make_float2(re[t], im[t]));
                        re[t] = w.x; im[t] = w.y;
                    }
                }
            if (g.mode == 1) {
                double2 *y = g.y + ((size_t)c * n + i) * n + jb;
#pragma unroll
                for (int t = 0; t < 16; ++t)
                    if (t < count) y[t] = make_double2(re[t], im[t]);
            } else {
                float *h = g.hi + ((size_t)c * n + i) * g.ld + 2 * jb;
                float *l = g.lo + ((size_t)c * n + i) * g.ld + 2 * jb;
                if (count == 16) {
#pragma unroll
                    for (int t = 0; t < 16; t += 2) {
                        float4 vh, vl;
                        vh.x = tf32_round(re[t]); vh.y = tf32_round(im[t]);
                        vh.z = tf32_round(re[t + 1]); vh.w = tf32_round(im[t + 1]);
                        vl.x = tf32_round(re[t] - vh.x); vl.y = tf32_round(im[t] - vh.y);
                        vl.z = tf32_round(re[t + 1] - vh.z); vl.w = tf32_round(im[t + 1] - vh.w);
                        *reinterpret_cast<float4 *>(h + 2 * t) = vh;
                        *reinterpret_cast<float4 *>(l + 2 * t) = vl;
                    }
                } else {
                    for (int t = 0; t < count; ++t) {
                        const float hr = tf32_round(re[t]), hi = tf32_round(im[t]);
                        h[2 * t] = hr; h[2 * t + 1] = hi;
                        l[2 * t] = tf32_round(re[t] - hr); l[2 * t + 1] = tf32_round(im[t] - hi);
                    }
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (lost && threadIdx.x == 0 && g.err) atomicExch(g.err, 1);
    if (warp == 2) tmem_free(tmem, TG_BN_MAX);
}

// complex128 x -> TF32 hi/lo planes, row (c n + j) of the plane = column j of Psi_c.
__global__ void split_tf32_kernel(size_t rows, int n, int ld, const double2 *__restrict__ x, float *__restrict__ hi,
                                  float *__restrict__ lo, const int *gate)
{
    if (gate && *gate) return;
    const size_t total = rows * (size_t)n;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
        const size_t r = p / n;
        const int k = (int)(p % n);
        const double2 v = x[p];
        const float vr = (float)v.x, vi = (float)v.y;
        const float hr = sm100::tf32_round(vr), hi_ = sm100::tf32_round(vi);
        float2 *h = reinterpret_cast<float2 *>(hi + r * ld) + k, *l = reinterpret_cast<float2 *>(lo + r * ld) + k;
        *h = make_float2(hr, hi_);
        *l = make_float2(sm100::tf32_round(vr - hr), sm100::tf32_round(vi - hi_));
    }
}

}  // namespace he

// ---------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------
using namespace he;

struct he_separable {
    int device = 0, n = 0, nc = 0, nl = 0, precision = 0, passes = 3;
    int tile = -1;                               // complex128 tile shape: -1 = default rule, else fixed
    int ld = 0, bn = 0, ntn = 0, kt = 0;         // complex64 GEMM geometry
    // complex128: S and S^-1 row-major (nl x n x n), two n^2 nc work vectors
    void *S = nullptr, *I = nullptr;
    void *evals = nullptr;                       // nl x n of the precision
    int *l1 = nullptr, *l2 = nullptr;            // per channel (device)
    void *buf[2] = {nullptr, nullptr};
    // complex64: embeddings of S and S^-1 (hi, lo), two pairs of hi/lo planes
    float *emb[4] = {nullptr, nullptr, nullptr, nullptr};   // S hi, S lo, I hi, I lo
    float *plane[4] = {nullptr, nullptr, nullptr, nullptr}; // pair 0 hi, lo; pair 1 hi, lo
    CUtensorMap mS[2], mI[2], mP0[2], mP1[2];
    int *err = nullptr;
    ~he_separable()
    {
        cudaFree(S); cudaFree(I); cudaFree(evals); cudaFree(l1); cudaFree(l2);
        cudaFree(buf[0]); cudaFree(buf[1]); cudaFree(err);
        for (float *p : emb) cudaFree(p);
        for (float *p : plane) cudaFree(p);
    }
};

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encoder()
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

// 2-D fp32 map over `rows` rows of `cols` values at a row stride of ld floats; box of
// 32 values x box_rows rows, 128-byte swizzle, zero fill outside the tensor.
bool encode(CUtensorMap *map, const float *base, int cols, long long rows, int ld, int box_rows)
{
    auto fn = encoder();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)TG_BK, (cuuint32_t)box_rows};
    cuuint32_t elem[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box, elem,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Round to the nearest TF32 value, ties away from zero (cvt.rna.tf32.f32 on the host).
float tf32_host(float x)
{
    uint32_t b;
    memcpy(&b, &x, 4);
    if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0x1000u) & 0xffffe000u;
    memcpy(&x, &b, 4);
    return x;
}

// Real embedding of nl complex matrices (column-major n x n, interleaved): row 2i+p,
// column 2k+q of matrix l at [(l 2n + 2i + p) ld + 2k + q]; TF32 hi and lo parts.
void embed(const double *mats, int nl, int n, int ld, std::vector<float> &hi, std::vector<float> &lo)
{
    const size_t rows = (size_t)nl * 2 * n;
    hi.assign(rows * ld, 0.f);
    lo.assign(rows * ld, 0.f);
    for (int l = 0; l < nl; ++l)
        for (int k = 0; k < n; ++k)
            for (int i = 0; i < n; ++i) {
                const size_t src = 2 * (((size_t)l * n + k) * n + i);
                const double re = mats[src], im = mats[src + 1];
                const double v[2][2] = {{re, -im}, {im, re}};
                for (int p = 0; p < 2; ++p)
                    for (int q = 0; q < 2; ++q) {
                        const size_t dst = ((size_t)l * 2 * n + 2 * i + p) * ld + 2 * k + q;
                        const float f = (float)v[p][q], h = tf32_host(f);
                        hi[dst] = h;
                        lo[dst] = tf32_host(f - h);
                    }
            }
}

template <int WM, int WN, int FM, int FN>
int dgemm_chain(he_separable *h, const double2 *x, double2 *y, double2 alpha, double shift, const int *gate,
                cudaStream_t s)
{
    const int n = h->n;
    const double2 *S = static_cast<const double2 *>(h->S), *I = static_cast<const double2 *>(h->I);
    double2 *b0 = static_cast<double2 *>(h->buf[0]), *b1 = static_cast<double2 *>(h->buf[1]);
    const void *kernel = (const void *)sep_dgemm_kernel<WM, WN, FM, FN>;
    constexpr size_t smem = dg_smem<WM, WN, FM, FN>();
    constexpr int BM = 8 * FM * WM, BN = 8 * FN * WN;
    HE_CUDA_TRY(he_smem_limit(kernel, smem));
    const dim3 grid((n + BM - 1) / BM, (n + BN - 1) / BN, h->nc);
    const int threads = 32 * WM * WN;
    Resolvent<double> none{nullptr, nullptr, nullptr, mk<double>(0, 0), 0.0, 0};
    Resolvent<double> rs{static_cast<const double2 *>(h->evals), h->l2, h->l1, alpha, shift, 1};
    // rows of the second product run over r2 (S_{l2}^-1), its columns over r1
    sep_dgemm_kernel<WM, WN, FM, FN><<<grid, threads, smem, s>>>(n, I, h->l1, x, b0, none, gate);
    sep_dgemm_kernel<WM, WN, FM, FN><<<grid, threads, smem, s>>>(n, I, h->l2, b0, b1, rs, gate);
    sep_dgemm_kernel<WM, WN, FM, FN><<<grid, threads, smem, s>>>(n, S, h->l1, b1, b0, none, gate);
    sep_dgemm_kernel<WM, WN, FM, FN><<<grid, threads, smem, s>>>(n, S, h->l2, b0, y, none, gate);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

// Default tile shape (measured on B200 at n = 560, nc = 43 and n = 132, nc = 17): 64 x 64
// tiles at two CTAs per SM (8 warps per SM, the first CTA's store overlapping the second's
// loads) once the grid fills a wave of them; below that, 32 x 32 tiles of four 16 x 16 warps,
// which give small problems several warps per SM.  SeparablePreconditioner.autotune times
// every shape per operator.
int apply_c128(he_separable *h, const double2 *x, double2 *y, double2 alpha, double shift, const int *gate,
               cudaStream_t s)
{
    int shape = h->tile;
    if (shape < 0) {
        const long long ctas64 = (long long)((h->n + 63) / 64) * ((h->n + 63) / 64) * h->nc;
        shape = ctas64 >= 2LL * sm_count(h->device) ? 2 : 4;
    }
    switch (shape) {
    case 0: return dgemm_chain<2, 4, 4, 4>(h, x, y, alpha, shift, gate, s);
    case 1: return dgemm_chain<2, 3, 4, 4>(h, x, y, alpha, shift, gate, s);
    case 2: return dgemm_chain<2, 2, 4, 4>(h, x, y, alpha, shift, gate, s);
    case 3: return dgemm_chain<1, 2, 4, 4>(h, x, y, alpha, shift, gate, s);
    default: return dgemm_chain<2, 2, 2, 2>(h, x, y, alpha, shift, gate, s);
    }
}

int apply_c64(he_separable *h, const double2 *x, double2 *y, double2 alpha, double shift, const int *gate,
              cudaStream_t s)
{
    const int n = h->n;
    HE_CUDA_TRY(he_smem_limit((const void *)sep_tf32_kernel, TG_SMEM));
    split_tf32_kernel<<<4 * 148, 256, 0, s>>>((size_t)n * h->nc, n, h->ld, x, h->plane[0], h->plane[1], gate);
    const dim3 grid((2 * n + TG_BM - 1) / TG_BM, h->ntn, h->nc);
    TcArgs g{};
    g.n = n; g.nc = h->nc; g.bn = h->bn; g.kt = h->kt; g.passes = h->passes; g.arows = 2 * n; g.ld = h->ld;
    g.err = h->err;
    g.gate = gate;
    g.rs = Resolvent<float>{nullptr, nullptr, nullptr, mk<float>(0, 0), 0.f, 0};
    auto run = [&](const CUtensorMap *m, const int *sel, const CUtensorMap *in, int out_pair, int mode,
                   Resolvent<float> rs) {
        g.sel = sel; g.mode = mode; g.rs = rs;
        g.hi = h->plane[2 * out_pair]; g.lo = h->plane[2 * out_pair + 1]; g.y = y;
        sep_tf32_kernel<<<grid, TG_THREADS, TG_SMEM, s>>>(m[0], m[1], in[0], in[1], g);
    };
    const Resolvent<float> none = g.rs;
    const Resolvent<float> rs{static_cast<const float2 *>(h->evals), h->l2, h->l1,
                              mk<float>((float)alpha.x, (float)alpha.y), (float)shift, 1};
    run(h->mI, h->l1, h->mP0, 1, 0, none);    // T = (I1 X)^T              pair 0 -> pair 1
    run(h->mI, h->l2, h->mP1, 0, 0, rs);      // Z = (I2 T)^T / resolvent  pair 1 -> pair 0
    run(h->mS, h->l1, h->mP0, 1, 0, none);    // T = (S1 Z)^T              pair 0 -> pair 1
    run(h->mS, h->l2, h->mP1, 0, 1, none);    // Y = (S2 T)^T              pair 1 -> y
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

}  // namespace

extern "C" int he_separable_create(he_separable **out, int n, int nc, int nl, const double *S, const double *Sinv,
                                   const double *evals, const int *l1, const int *l2, int precision)
{
    if (!out || !S || !Sinv || !evals || !l1 || !l2 || n < 1 || nc < 1 || nl < 1)
        return he_fail(HE_ERR_ARG, "bad separable preconditioner argument", __FILE__, __LINE__);
    if (precision != HE_C128 && precision != HE_C64) return he_fail(HE_ERR_ARG, "bad precision", __FILE__, __LINE__);
    for (int c = 0; c < nc; ++c)
        if (l1[c] < 0 || l1[c] >= nl || l2[c] < 0 || l2[c] >= nl)
            return he_fail(HE_ERR_SHAPE, "channel angular momentum outside the eigenbasis table", __FILE__, __LINE__);
    *out = nullptr;
    he_separable *h = new he_separable();
    h->n = n; h->nc = nc; h->nl = nl; h->precision = precision;
    const size_t nn = (size_t)n * n;
    auto fail = [&](cudaError_t e) { he_set_error(cudaGetErrorString(e), __FILE__, __LINE__); delete h; return HE_ERR_CUDA; };
    cudaError_t e = cudaGetDevice(&h->device);
    auto copy = [&](void **dst, const void *src, size_t bytes) -> cudaError_t {
        cudaError_t r = cudaMalloc(dst, bytes);
        return r != cudaSuccess ? r : cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    };
    if (e == cudaSuccess) e = copy((void **)&h->l1, l1, nc * sizeof(int));
    if (e == cudaSuccess) e = copy((void **)&h->l2, l2, nc * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&h->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->err, 0, sizeof(int));
    if (precision == HE_C128) {
        // column-major (the caller's layout) -> row-major for the K-contiguous A tiles
        std::vector<double2> rm(nl * nn);
        auto transpose = [&](const double *src) {
            for (int l = 0; l < nl; ++l)
                for (int k = 0; k < n; ++k)
                    for (int i = 0; i < n; ++i) {
                        const size_t a = 2 * (((size_t)l * n + k) * n + i);
                        rm[((size_t)l * n + i) * n + k] = make_double2(src[a], src[a + 1]);
                    }
        };
        transpose(S);
        if (e == cudaSuccess) e = copy(&h->S, rm.data(), rm.size() * sizeof(double2));
        transpose(Sinv);
        if (e == cudaSuccess) e = copy(&h->I, rm.data(), rm.size() * sizeof(double2));
        if (e == cudaSuccess) e = copy(&h->evals, evals, (size_t)nl * n * sizeof(double2));
        if (e == cudaSuccess) e = cudaMalloc(&h->buf[0], nn * nc * sizeof(double2));
        if (e == cudaSuccess) e = cudaMalloc(&h->buf[1], nn * nc * sizeof(double2));
        if (e != cudaSuccess) return fail(e);
    } else {
        h->ld = (2 * n + 3) / 4 * 4;                       // 16-byte row stride for TMA
        h->kt = (2 * n + TG_BK - 1) / TG_BK;
        // N tiles: as few as the 256 TMEM columns allow, more when the grid would leave SMs idle
        const int mtiles = (2 * n + TG_BM - 1) / TG_BM;
        h->ntn = (n + TG_BN_MAX - 1) / TG_BN_MAX;
        const int fill = (sm_count(h->device) + mtiles * nc - 1) / (mtiles * nc);
        h->ntn = std::max(h->ntn, std::min(fill, std::max(1, n / 32)));
        h->bn = ((n + h->ntn - 1) / h->ntn + 15) / 16 * 16;
        h->ntn = (n + h->bn - 1) / h->bn;
        std::vector<float2> ev((size_t)nl * n);
        for (size_t k = 0; k < ev.size(); ++k) ev[k] = make_float2((float)evals[2 * k], (float)evals[2 * k + 1]);
        if (e == cudaSuccess) e = copy(&h->evals, ev.data(), ev.size() * sizeof(float2));
        std::vector<float> hi, lo;
        const size_t ebytes = (size_t)nl * 2 * n * h->ld * sizeof(float);
        embed(S, nl, n, h->ld, hi, lo);
        if (e == cudaSuccess) e = copy((void **)&h->emb[0], hi.data(), ebytes);
        if (e == cudaSuccess) e = copy((void **)&h->emb[1], lo.data(), ebytes);
        embed(Sinv, nl, n, h->ld, hi, lo);
        if (e == cudaSuccess) e = copy((void **)&h->emb[2], hi.data(), ebytes);
        if (e == cudaSuccess) e = copy((void **)&h->emb[3], lo.data(), ebytes);
        const size_t pbytes = (size_t)n * nc * h->ld * sizeof(float);
        for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
            e = cudaMalloc((void **)&h->plane[k], pbytes);
            if (e == cudaSuccess) e = cudaMemset(h->plane[k], 0, pbytes);   // the row padding stays zero
        }
        if (e != cudaSuccess) return fail(e);
        const long long arows = (long long)nl * 2 * n, xrows = (long long)n * nc;
        const bool ok = encode(&h->mS[0], h->emb[0], 2 * n, arows, h->ld, TG_BM) &&
                        encode(&h->mS[1], h->emb[1], 2 * n, arows, h->ld, TG_BM) &&
                        encode(&h->mI[0], h->emb[2], 2 * n, arows, h->ld, TG_BM) &&
                        encode(&h->mI[1], h->emb[3], 2 * n, arows, h->ld, TG_BM) &&
                        encode(&h->mP0[0], h->plane[0], 2 * n, xrows, h->ld, h->bn) &&
                        encode(&h->mP0[1], h->plane[1], 2 * n, xrows, h->ld, h->bn) &&
                        encode(&h->mP1[0], h->plane[2], 2 * n, xrows, h->ld, h->bn) &&
                        encode(&h->mP1[1], h->plane[3], 2 * n, xrows, h->ld, h->bn);
        if (!ok) { delete h; return he_fail(HE_ERR_CUDA, "cuTensorMapEncodeTiled failed", __FILE__, __LINE__); }
    }
    *out = h;
    return HE_OK;
}

extern "C" int he_separable_destroy(he_separable *h)
{
    delete h;
    return HE_OK;
}

// Number of TF32 products per K slice of the complex64 GEMMs: 3 (split operands, FP32-class
// accuracy, the default) or 1 (TF32 operands only).
extern "C" int he_separable_set_passes(he_separable *h, int passes)
{
    if (!h || (passes != 1 && passes != 3)) return he_fail(HE_ERR_ARG, "passes must be 1 or 3", __FILE__, __LINE__);
    h->passes = passes;
    return HE_OK;
}

// Tile shape of the complex128 GEMMs: 0 = 64 x 128, 1 = 64 x 96, 2 = 64 x 64, 3 = 32 x 64
// (32 x 32 per warp), 4 = 32 x 32 (16 x 16 per warp) outputs per CTA, -1 = the default rule
// of apply_c128.
extern "C" int he_separable_set_tile(he_separable *h, int shape)
{
    if (!h || shape < -1 || shape > 4) return he_fail(HE_ERR_ARG, "tile shape must be -1..4", __FILE__, __LINE__);
    h->tile = shape;
    return HE_OK;
}

// Device error word of the complex64 GEMMs (a bounded wait that ran out); read and cleared.
extern "C" int he_separable_status(he_separable *h)
{
    if (!h) return he_fail(HE_ERR_ARG, "null preconditioner", __FILE__, __LINE__);
    int v = 0;
    HE_CUDA_TRY(cudaMemcpy(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (v) {
        HE_CUDA_TRY(cudaMemset(h->err, 0, sizeof(int)));
        return he_fail(HE_ERR_DEVICE, "separable preconditioner: a pipeline wait ran out", __FILE__, __LINE__);
    }
    return HE_OK;
}

// y = M(alpha, shift) x ; x, y complex128 device vectors of n*n*nc elements (y != x).
extern "C" int he_separable_apply(he_separable *h, const void *x, void *y, double alpha_re, double alpha_im,
                                  double shift, void *stream)
{
    if (!h || !x || !y || x == y) return he_fail(HE_ERR_ARG, "bad separable apply argument", __FILE__, __LINE__);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    return he::separable_apply_gated(h, static_cast<const double2 *>(x), static_cast<double2 *>(y),
                                     mk<double>(alpha_re, alpha_im), shift, nullptr, s);
}

// The same apply whose kernels return without work while *gate != 0 (the GMRES driver's
// gate words; gate may be null).
int he::separable_apply_gated(he_separable *h, const double2 *x, double2 *y, double2 alpha, double shift,
                              const int *gate, cudaStream_t s)
{
    if (h->precision == HE_C128) return apply_c128(h, x, y, alpha, shift, gate, s);
    return apply_c64(h, x, y, alpha, shift, gate, s);
}
