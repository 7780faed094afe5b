// Online tSURFF on the device, complex128 throughout:
//
//   he_surface_contract  q[j, o, s] = sum_{c : outer(j,c) = o} coef(j,c)
//                                     sum_r conj(chi[inner(j,c), r, column(j)]) frame(r, s, c)
//                        — the ionic contraction of python/surface_contract.py:41-56 in a
//                        table form that covers its product-basis and coupled ("fast")
//                        paths (tables built on the host by laqphysics_b200.surface_contract);
//   he_volkov_add        amplitude += d (previous + current) / 2,
//                        current[j,e,a] = i sqrt(2) phase(e,a) sum_l harmonics[l,a]
//                                         sum_s q[j,l,s] tests[l,e,s],
//                        phase = exp(i (E t + k (u_a . int A) + int A^2 / 2))
//                        — python/streaming_surface.py:54-64 (and its GPU twin :97-109);
//   he_sample_record     one surface sample in ONE launch: the flux frame of the state
//                        (he_flux's arithmetic), the contraction and the Volkov update —
//                        the chain python/streaming_surface.py:252-255 runs per sample.
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "operator.cuh"

namespace he {

constexpr int SURF_THREADS = 256;

// One CTA per (label j, outer o, surface row s); entries of label j are
// (frame column, inner ionic state, real coefficient, outer state).
__global__ void __launch_bounds__(SURF_THREADS)
surface_contract_kernel(long long n, int nunique, int nouter, int ns, const double2 *__restrict__ chi,
                        const double2 *__restrict__ frame, long long fr, long long fs, long long fc,
                        const int *__restrict__ eptr, const int *__restrict__ ecol, const int *__restrict__ einner,
                        const double *__restrict__ ecoef, const int *__restrict__ eouter, const int *__restrict__ column,
                        double2 *__restrict__ q)
{
    const int s = blockIdx.x % ns;
    const int o = (blockIdx.x / ns) % nouter;
    const int j = blockIdx.x / (ns * nouter);
    const int col = column[j];
    double2 acc = mk<double>(0, 0);
    for (int e = eptr[j]; e < eptr[j + 1]; ++e) {
        if (eouter[e] != o) continue;
        const double w = ecoef[e];
        const size_t a = (size_t)einner[e];
        const long long c = ecol[e];
        double2 part = mk<double>(0, 0);
        for (long long r = threadIdx.x; r < n; r += blockDim.x) {
            const double2 x = chi[(a * n + r) * nunique + col];
            part = cfma_conj<double>(x, frame[r * fr + (long long)s * fs + c * fc], part);
        }
        acc = rfma<double>(w, part, acc);
    }
    __shared__ double2 red[SURF_THREADS / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        acc.x += __shfl_down_sync(0xffffffffu, acc.x, off);
        acc.y += __shfl_down_sync(0xffffffffu, acc.y, off);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = mk<double>(0, 0);
        for (int w = 0; w < SURF_THREADS / 32; ++w) t = cadd<double>(t, red[w]);
        q[((size_t)j * nouter + o) * ns + s] = t;
    }
}

// Volkov item idx = (label j, energy e, direction a): current = i sqrt(2) phase sum_l
// harm[l, a] sum_s q[j, l, s] tests[l, e, s]; trapezoid update of the amplitude.
__device__ __forceinline__ void volkov_item(long long idx, int nouter, int ns, int ne, int nang,
                                            const double2 *__restrict__ q, const double2 *__restrict__ tests,
                                            const double2 *__restrict__ harm, const double *__restrict__ energy,
                                            const double *__restrict__ k, const double *__restrict__ unit, double time,
                                            double ax, double ay, double az, double a2, double d, int first,
                                            double2 *__restrict__ amplitude, double2 *__restrict__ previous)
{
    const int a = (int)(idx % nang);
    const int e = (int)((idx / nang) % ne);
    const int j = (int)(idx / ((long long)nang * ne));
    double2 sum = mk<double>(0, 0);
    for (int l = 0; l < nouter; ++l) {
        double2 radial = mk<double>(0, 0);
        const double2 *ql = q + ((size_t)j * nouter + l) * ns;
        const double2 *tl = tests + ((size_t)l * ne + e) * ns;
        for (int s = 0; s < ns; ++s) radial = cfma<double>(ql[s], tl[s], radial);
        sum = cfma<double>(radial, harm[(size_t)l * nang + a], sum);
    }
    const double disp = unit[3 * a] * ax + unit[3 * a + 1] * ay + unit[3 * a + 2] * az;
    const double arg = energy[e] * time + k[e] * disp + a2 / 2;
    double sn, cs;
    sincos(arg, &sn, &cs);
    // current = i sqrt(2) sum * exp(i arg)
    const double2 ph = mk<double>(cs, sn);
    const double2 t = cmul<double>(sum, ph);
    const double r2 = sqrt(2.0);
    const double2 cur = mk<double>(-r2 * t.y, r2 * t.x);
    const size_t o = (size_t)idx;
    if (!first) {
        const double2 prev = previous[o];
        amplitude[o] = rfma<double>(d / 2, cadd<double>(prev, cur), amplitude[o]);
    }
    previous[o] = cur;
}

__global__ void __launch_bounds__(SURF_THREADS)
volkov_add_kernel(int nlab, int nouter, int ns, int ne, int nang, const double2 *__restrict__ q,
                  const double2 *__restrict__ tests, const double2 *__restrict__ harm, const double *__restrict__ energy,
                  const double *__restrict__ k, const double *__restrict__ unit, double time, double ax, double ay,
                  double az, double a2, double d, int first, double2 *__restrict__ amplitude,
                  double2 *__restrict__ previous)
{
    const long long total = (long long)nlab * ne * nang;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x)
        volkov_item(idx, nouter, ns, ne, nang, q, tests, harm, energy, k, unit, time, ax, ay, az, a2, d, first,
                    amplitude, previous);
}

// ---- one launch per surface sample -------------------------------------------------
// A cooperative grid (every CTA resident) in three phases:
//  1. tiles of 32 radial rows x 8 channels: the flux frame rows of the tile (written out,
//     and kept in shared memory), then the tile's share of every q entry (warp w owns the
//     (label, outer state) pairs w, w + 8, ... with all their surface rows; lanes run over
//     the tile's radial rows), summed per CTA;
//  2. each CTA that had tiles stores its partial q; all arrive on a counter and wait
//     (bounded) for all;
//  3. each q entry is summed once over those partials in CTA order (reproducible bit for
//     bit) by the CTA it falls to and stored; a second wait on the same counter; every CTA
//     reads q and the CTAs share the Volkov items.
constexpr int SAMPLE_THREADS = 256, SAMPLE_TA = 32, SAMPLE_TC = SAMPLE_THREADS / SAMPLE_TA;
constexpr int SAMPLE_NS_MAX = 16, SAMPLE_NQ_MAX = 1024;
constexpr int SAMPLE_SC = 8;                     // surface rows held in registers at a time
constexpr int SAMPLE_WAIT_LIMIT = 1 << 20;   // polls of the arrival counter (about a second)

struct SampleArgs {
    DeviceTables<double> t;                  // n, nc and the dipole edges of the operator
    const double2 *psi;
    double2 *frame;                          // (c, s, r): frame[r + n (s + ns c)], as he_flux
    int ns, lo, width;
    const double2 *J, *JP;
    double f0, f1, f2;
    const double2 *chi;
    int nunique, nlab, nouter;
    const int *eptr, *ecol, *einner, *eouter, *column;
    const double *ecoef;
    double2 *q;
    int ne, nang;
    const double2 *tests, *harm;
    const double *energy, *k, *unit;
    double time, ax, ay, az, a2, d;
    int first;
    double2 *amplitude, *previous;
    double2 *partial;                        // gridDim.x x nq
    unsigned *arrived;                       // zeroed before the launch
    unsigned extra;                          // arrivals awaited beyond the grid (0; a test hook)
    int *err;
};

// Arrive on the counter and wait (thread 0, bounded) until it reaches `target`; false, with
// the error word set, when the wait ran out.  Every thread of the CTA calls it.
__device__ bool sample_grid_wait(unsigned *arrived, unsigned target, int *err, volatile int &lost)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(arrived, 1u);
        bool ok = false;
        for (int k = 0; k < SAMPLE_WAIT_LIMIT && !ok; ++k) {
            ok = *reinterpret_cast<volatile unsigned *>(arrived) >= target;
            if (!ok) __nanosleep(256);
        }
        __threadfence();
        if (!ok) {
            lost = 1;
            atomicExch(err, 1);
        }
    }
    __syncthreads();
    return !lost;
}

__global__ void __launch_bounds__(SAMPLE_THREADS) surface_sample_kernel(const __grid_constant__ SampleArgs g)
{
    extern __shared__ __align__(16) unsigned char sample_smem[];
    __shared__ volatile int lost;
    const int n = g.t.n, nc = g.t.nc, ns = g.ns;
    const int nq = g.nlab * g.nouter * ns;
    double2 *F = reinterpret_cast<double2 *>(sample_smem);          // [ns][SAMPLE_TC][SAMPLE_TA]
    double2 *Q = F + (size_t)ns * SAMPLE_THREADS;                   // [nq]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int al = tid % SAMPLE_TA, cl = tid / SAMPLE_TA;
    const size_t nn = (size_t)n * n;
    const int tiles_a = (n + SAMPLE_TA - 1) / SAMPLE_TA, tiles = tiles_a * ((nc + SAMPLE_TC - 1) / SAMPLE_TC);
    if (tid == 0) lost = 0;
    for (int i = tid; i < nq; i += SAMPLE_THREADS) Q[i] = mk<double>(0, 0);
    __syncthreads();
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int a0 = (tile % tiles_a) * SAMPLE_TA, c0 = (tile / tiles_a) * SAMPLE_TC;
        const int a = a0 + al, c = c0 + cl;
        // flux frame rows of (a, c), eight surface rows at a time: each psi value of the
        // window is read once per chunk; per row the operations of flux_kernel, in its order
        for (int s0 = 0; s0 < ns; s0 += SAMPLE_SC) {
            double2 acc[SAMPLE_SC];
#pragma unroll
            for (int u = 0; u < SAMPLE_SC; ++u) acc[u] = mk<double>(0, 0);
            if (a < n && c < nc) {
                const double2 *pc = g.psi + nn * c + a;
                for (int q = 0; q < g.width; ++q) {
                    const double2 x = pc[(size_t)n * (g.lo + q)];
#pragma unroll
                    for (int u = 0; u < SAMPLE_SC; ++u)
                        if (s0 + u < ns) acc[u] = cfma<double>(ldg<double>(g.J + (size_t)(s0 + u) * g.width + q), x, acc[u]);
                }
                for (int k = __ldg(g.t.dptr + c), e = __ldg(g.t.dptr + c + 1); k < e; ++k) {
                    if (__ldg(g.t.de + k) != 2) continue;
                    const double2 *dk = g.t.dcoef + 3 * (size_t)k;
                    double2 coef = cscale<double>(g.f0, ldg<double>(dk));
                    coef = rfma<double>(g.f1, ldg<double>(dk + 1), coef);
                    coef = rfma<double>(g.f2, ldg<double>(dk + 2), coef);
                    if (sqrt(cabs2<double>(coef)) <= 1e-15) continue;
                    const double2 *ps = g.psi + nn * __ldg(g.t.dc + k) + a;
                    double2 part[SAMPLE_SC];
#pragma unroll
                    for (int u = 0; u < SAMPLE_SC; ++u) part[u] = mk<double>(0, 0);
                    for (int q = 0; q < g.width; ++q) {
                        const double2 y = ps[(size_t)n * (g.lo + q)];
#pragma unroll
                        for (int u = 0; u < SAMPLE_SC; ++u)
                            if (s0 + u < ns)
                                part[u] = cfma<double>(ldg<double>(g.JP + (size_t)(s0 + u) * g.width + q), y, part[u]);
                    }
#pragma unroll
                    for (int u = 0; u < SAMPLE_SC; ++u)
                        if (s0 + u < ns) acc[u] = cfma<double>(coef, part[u], acc[u]);
                }
#pragma unroll
                for (int u = 0; u < SAMPLE_SC; ++u)
                    if (s0 + u < ns) g.frame[a + (size_t)n * (s0 + u + (size_t)ns * c)] = acc[u];
            }
#pragma unroll
            for (int u = 0; u < SAMPLE_SC; ++u)
                if (s0 + u < ns) F[((s0 + u) * SAMPLE_TC + cl) * SAMPLE_TA + al] = acc[u];
        }
        __syncthreads();
        // contraction partials of this tile: warp w owns the (label, outer) pairs w, w + 8, ...
        // and with them the q entries of all their surface rows; each entry of a pair is read
        // once per chunk of eight rows
        for (int jo = warp; jo < g.nlab * g.nouter; jo += SAMPLE_THREADS / 32) {
            const int j = jo / g.nouter, o = jo % g.nouter;
            const size_t col = (size_t)g.column[j];
            for (int s0 = 0; s0 < ns; s0 += SAMPLE_SC) {
                double2 acc[SAMPLE_SC];
#pragma unroll
                for (int u = 0; u < SAMPLE_SC; ++u) acc[u] = mk<double>(0, 0);
                for (int e = g.eptr[j]; e < g.eptr[j + 1]; ++e) {
                    const int ce = g.ecol[e];
                    if (g.eouter[e] != o || ce < c0 || ce >= c0 + SAMPLE_TC) continue;
                    const double w = g.ecoef[e];
                    const double2 x = a0 + lane < n ? g.chi[((size_t)g.einner[e] * n + a0 + lane) * g.nunique + col]
                                                    : mk<double>(0, 0);
#pragma unroll
                    for (int u = 0; u < SAMPLE_SC; ++u) {
                        if (s0 + u >= ns) continue;
                        double2 part = mk<double>(0, 0);
                        if (a0 + lane < n)
                            part = cfma_conj<double>(x, F[((s0 + u) * SAMPLE_TC + (ce - c0)) * SAMPLE_TA + lane], part);
                        acc[u] = rfma<double>(w, part, acc[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < SAMPLE_SC; ++u) {
                    if (s0 + u >= ns) continue;
                    double2 v = acc[u];
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) {
                        v.x += __shfl_down_sync(0xffffffffu, v.x, off);
                        v.y += __shfl_down_sync(0xffffffffu, v.y, off);
                    }
                    if (lane == 0) Q[jo * ns + s0 + u] = cadd<double>(Q[jo * ns + s0 + u], v);
                }
            }
        }
        __syncthreads();
    }
    // CTAs past the last tile hold no partial sums
    const int with_tiles = (int)gridDim.x < tiles ? (int)gridDim.x : tiles;
    if ((int)blockIdx.x < with_tiles)
        for (int i = tid; i < nq; i += SAMPLE_THREADS) g.partial[(size_t)blockIdx.x * nq + i] = Q[i];
    // every CTA's partials, then each q entry summed once (in CTA order, by the CTA and
    // thread it falls to), then every CTA reads q
    if (!sample_grid_wait(g.arrived, gridDim.x + g.extra, g.err, lost)) return;
    for (int i = (int)blockIdx.x + (int)gridDim.x * tid; i < nq; i += (int)gridDim.x * SAMPLE_THREADS) {
        double2 v = mk<double>(0, 0);
        for (int b = 0; b < with_tiles; ++b) v = cadd<double>(v, __ldcg(g.partial + (size_t)b * nq + i));
        g.q[i] = v;
    }
    if (!sample_grid_wait(g.arrived, 2 * gridDim.x + g.extra, g.err, lost)) return;
    for (int i = tid; i < nq; i += SAMPLE_THREADS) Q[i] = __ldcg(g.q + i);
    __syncthreads();
    const long long total = (long long)g.nlab * g.ne * g.nang;
    for (long long idx = blockIdx.x * (long long)SAMPLE_THREADS + tid; idx < total;
         idx += (long long)gridDim.x * SAMPLE_THREADS)
        volkov_item(idx, g.nouter, ns, g.ne, g.nang, Q, g.tests, g.harm, g.energy, g.k, g.unit, g.time, g.ax, g.ay,
                    g.az, g.a2, g.d, g.first, g.amplitude, g.previous);
}

}  // namespace he

using namespace he;

extern "C" int he_surface_contract(long long n, int nunique, int nlab, int nouter, int ns, const void *chi,
                                   const void *frame, long long fr, long long fs, long long fc, const int *eptr,
                                   const int *ecol, const int *einner, const double *ecoef, const int *eouter,
                                   const int *column, void *q, void *stream)
{
    if (n < 1 || nunique < 1 || nlab < 1 || nouter < 1 || ns < 1 || !chi || !frame || !eptr || !ecol || !einner ||
        !ecoef || !eouter || !column || !q)
        return he_fail(HE_ERR_ARG, "bad surface contraction argument", __FILE__, __LINE__);
    surface_contract_kernel<<<nlab * nouter * ns, SURF_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(
        n, nunique, nouter, ns, static_cast<const double2 *>(chi), static_cast<const double2 *>(frame), fr, fs, fc,
        eptr, ecol, einner, ecoef, eouter, column, static_cast<double2 *>(q));
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

extern "C" int he_volkov_add(int nlab, int nouter, int ns, int ne, int nang, const void *q, const void *tests,
                             const void *harmonics, const double *energy, const double *k, const double *unit,
                             double time, const double *int_a, double int_a2, double d, int first, void *amplitude,
                             void *previous, void *stream)
{
    if (nlab < 1 || nouter < 1 || ns < 1 || ne < 1 || nang < 1 || !q || !tests || !harmonics || !energy || !k ||
        !unit || !int_a || !amplitude || !previous)
        return he_fail(HE_ERR_ARG, "bad Volkov accumulator argument", __FILE__, __LINE__);
    const long long total = (long long)nlab * ne * nang;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 1184);
    volkov_add_kernel<<<blocks, SURF_THREADS, 0, static_cast<cudaStream_t>(stream)>>>(
        nlab, nouter, ns, ne, nang, static_cast<const double2 *>(q), static_cast<const double2 *>(tests),
        static_cast<const double2 *>(harmonics), energy, k, unit, time, int_a[0], int_a[1], int_a[2], int_a2, d, first,
        static_cast<double2 *>(amplitude), static_cast<double2 *>(previous));
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}

// ---- fused surface sample ------------------------------------------------------------
struct he_sample {
    int device = 0;
    he::SampleArgs args{};                   // the tables; per-sample fields are set by he_sample_record
    int grid = 0;
    size_t smem = 0;
    double2 *partial = nullptr;
    unsigned *arrived = nullptr;
    int *err = nullptr;
    ~he_sample()
    {
        cudaFree(partial);
        cudaFree(arrived);
        cudaFree(err);
    }
};

extern "C" int he_sample_create(he_sample **out, he_handle op, int ns, int lo, int width, const void *J,
                                const void *JP, int nunique, int nlab, int nouter, const int *eptr, const int *ecol,
                                const int *einner, const double *ecoef, const int *eouter, const int *column, int ne,
                                int nang, const void *tests, const void *harmonics, const double *energy,
                                const double *k, const double *unit)
{
    if (!out || !op || !J || !JP || !eptr || !ecol || !einner || !ecoef || !eouter || !column || !tests || !harmonics ||
        !energy || !k || !unit || nunique < 1 || nlab < 1 || nouter < 1 || ne < 1 || nang < 1)
        return he_fail(HE_ERR_ARG, "bad surface sample argument", __FILE__, __LINE__);
    if (ns < 1 || ns > SAMPLE_NS_MAX || width < 1 || lo < 0 || lo + width > op->n)
        return he_fail(HE_ERR_SHAPE, "surface stencil outside the grid or more than 16 surface rows", __FILE__,
                       __LINE__);
    const int nq = nlab * nouter * ns;
    if (nq > SAMPLE_NQ_MAX)
        return he_fail(HE_ERR_SHAPE, "more than 1024 contracted surface values per sample", __FILE__, __LINE__);
    *out = nullptr;
    int device = 0;
    HE_CUDA_TRY(cudaGetDevice(&device));
    he_sample *h = new he_sample();
    h->device = device;
    SampleArgs &a = h->args;
    a.t = op->t64;
    a.ns = ns; a.lo = lo; a.width = width;
    a.J = static_cast<const double2 *>(J); a.JP = static_cast<const double2 *>(JP);
    a.nunique = nunique; a.nlab = nlab; a.nouter = nouter;
    a.eptr = eptr; a.ecol = ecol; a.einner = einner; a.eouter = eouter; a.column = column; a.ecoef = ecoef;
    a.ne = ne; a.nang = nang;
    a.tests = static_cast<const double2 *>(tests); a.harm = static_cast<const double2 *>(harmonics);
    a.energy = energy; a.k = k; a.unit = unit;
    h->smem = ((size_t)ns * SAMPLE_THREADS + nq) * sizeof(double2);
    const int tiles = ((op->n + SAMPLE_TA - 1) / SAMPLE_TA) * ((op->nc + SAMPLE_TC - 1) / SAMPLE_TC);
    const long long items = ((long long)nlab * ne * nang + SAMPLE_THREADS - 1) / SAMPLE_THREADS;
    const cudaError_t limit = he_smem_limit(reinterpret_cast<const void *>(surface_sample_kernel), h->smem);
    if (limit != cudaSuccess) {
        he_set_error(cudaGetErrorString(limit), __FILE__, __LINE__);
        delete h;
        return HE_ERR_CUDA;
    }
    const int resident = resident_ctas(reinterpret_cast<const void *>(surface_sample_kernel), SAMPLE_THREADS, h->smem) *
                         sm_count(h->device);
    h->grid = (int)std::max<long long>(1, std::min<long long>(resident, std::max<long long>(tiles, items)));
    auto fail = [&](cudaError_t e) {
        he_set_error(cudaGetErrorString(e), __FILE__, __LINE__);
        delete h;
        return HE_ERR_CUDA;
    };
    cudaError_t e = cudaMalloc(&h->partial, (size_t)h->grid * nq * sizeof(double2));
    if (e == cudaSuccess) e = cudaMalloc(&h->arrived, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&h->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->err, 0, sizeof(int));
    if (e != cudaSuccess) return fail(e);
    a.partial = h->partial; a.arrived = h->arrived; a.err = h->err;
    *out = h;
    return HE_OK;
}

extern "C" int he_sample_record(he_sample *h, const void *psi, const void *chi, const double *field, double time,
                                const double *int_a, double int_a2, double d, int first, void *frame, void *q,
                                void *amplitude, void *previous, void *stream)
{
    if (!h || !psi || !chi || !field || !int_a || !frame || !q || !amplitude || !previous)
        return he_fail(HE_ERR_ARG, "null surface sample argument", __FILE__, __LINE__);
    SampleArgs a = h->args;
    a.psi = static_cast<const double2 *>(psi);
    a.chi = static_cast<const double2 *>(chi);
    a.f0 = field[0]; a.f1 = field[1]; a.f2 = field[2];
    a.time = time; a.ax = int_a[0]; a.ay = int_a[1]; a.az = int_a[2]; a.a2 = int_a2; a.d = d; a.first = first;
    a.frame = static_cast<double2 *>(frame);
    a.q = static_cast<double2 *>(q);
    a.amplitude = static_cast<double2 *>(amplitude);
    a.previous = static_cast<double2 *>(previous);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    HE_CUDA_TRY(he_smem_limit(reinterpret_cast<const void *>(surface_sample_kernel), h->smem));
    HE_CUDA_TRY(cudaMemsetAsync(h->arrived, 0, sizeof(unsigned), s));
    void *params[] = {&a};
    HE_CUDA_TRY(cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(surface_sample_kernel), dim3(h->grid),
                                            dim3(SAMPLE_THREADS), params, h->smem, s));
    return HE_OK;
}

extern "C" int he_sample_grid(he_sample *h) { return h ? h->grid : 0; }

// Test hook: the CTAs of later records wait for `extra` arrivals beyond the grid, which never
// come, so their bounded wait runs out (he_sample_status then reports it); 0 restores.
extern "C" int he_sample_set_wait_extra(he_sample *h, unsigned extra)
{
    if (!h) return he_fail(HE_ERR_ARG, "null surface sample", __FILE__, __LINE__);
    h->args.extra = extra;
    return HE_OK;
}

extern "C" int he_sample_status(he_sample *h)
{
    if (!h) return he_fail(HE_ERR_ARG, "null surface sample", __FILE__, __LINE__);
    int v = 0;
    HE_CUDA_TRY(cudaMemcpy(&v, h->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!v) return HE_OK;
    HE_CUDA_TRY(cudaMemset(h->err, 0, sizeof(int)));
    return he_fail(HE_ERR_DEVICE, "surface sample: the wait for every CTA's partial sums ran out", __FILE__, __LINE__);
}

extern "C" int he_sample_destroy(he_sample *h)
{
    delete h;
    return HE_OK;
}
