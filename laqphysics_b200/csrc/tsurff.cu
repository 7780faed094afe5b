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
//                        — python/streaming_surface.py:54-64 (and its GPU twin :97-109).
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

__global__ void __launch_bounds__(SURF_THREADS)
volkov_add_kernel(int nlab, int nouter, int ns, int ne, int nang, const double2 *__restrict__ q,
                  const double2 *__restrict__ tests, const double2 *__restrict__ harm, const double *__restrict__ energy,
                  const double *__restrict__ k, const double *__restrict__ unit, double time, double ax, double ay,
                  double az, double a2, double d, int first, double2 *__restrict__ amplitude,
                  double2 *__restrict__ previous)
{
    const long long total = (long long)nlab * ne * nang;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
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
