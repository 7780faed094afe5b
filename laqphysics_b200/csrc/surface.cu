// tSURFF surface flux frame on the device.
//
// frame(a, s, c) = sum_b J(s, b) psi(a, b, c)
//                + sum_{electron-2 dipole edges k of c} coef_k sum_b JP(s, b) psi(a, b, dc_k)
// with J the rows of the discrete commutator [H, Theta(r2 - R)] on the surface
// stencil and JP = i [T, Theta] (r_b - r_a) its velocity-gauge part
// (python/helium3d.py:52-77, python/torch_backend.py:133-138).  Only the nonzero
// column window [lo, lo + width) of the stencil rows is stored (width <= 64).
#include "common.cuh"
#include "operator.cuh"

namespace he {

template <typename R>
__global__ void __launch_bounds__(256)
flux_kernel(const DeviceTables<R> t, const cplx<R> *__restrict__ psi, cplx<R> *__restrict__ frame, int ns, int lo,
            int width, const cplx<R> *__restrict__ J, const cplx<R> *__restrict__ JP, R f0, R f1, R f2)
{
    const int n = t.n;
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    const int c = blockIdx.z;
    if (a >= n) return;
    const size_t nn = (size_t)n * n;
    const cplx<R> *pc = psi + nn * c + a;
    cplx<R> acc = mk<R>(0, 0);
    for (int q = 0; q < width; ++q) acc = cfma<R>(ldg<R>(J + (size_t)s * width + q), pc[(size_t)n * (lo + q)], acc);
    for (int k = __ldg(t.dptr + c), e = __ldg(t.dptr + c + 1); k < e; ++k) {
        if (__ldg(t.de + k) != 2) continue;
        const cplx<R> *dk = t.dcoef + 3 * (size_t)k;
        cplx<R> coef = cscale<R>(f0, ldg<R>(dk));
        coef = rfma<R>(f1, ldg<R>(dk + 1), coef);
        coef = rfma<R>(f2, ldg<R>(dk + 2), coef);
        if (sqrt(cabs2<R>(coef)) <= (R)1e-15) continue;
        const cplx<R> *ps = psi + nn * __ldg(t.dc + k) + a;
        cplx<R> part = mk<R>(0, 0);
        for (int q = 0; q < width; ++q)
            part = cfma<R>(ldg<R>(JP + (size_t)s * width + q), ps[(size_t)n * (lo + q)], part);
        acc = cfma<R>(coef, part, acc);
    }
    frame[a + (size_t)n * (s + (size_t)ns * c)] = acc;
}

}  // namespace he

extern "C" int he_flux(he_handle h, const void *psi, void *frame, int ns, int lo, int width, const void *J,
                       const void *JP, const double *field, void *stream)
{
    if (!h || !psi || !frame || !J || !JP || !field) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (ns < 1 || width < 1 || lo < 0 || lo + width > h->n)
        return he_fail(HE_ERR_SHAPE, "surface stencil outside the grid", __FILE__, __LINE__);
    const dim3 block(128);
    const dim3 grid((h->n + 127) / 128, ns, h->nc);
    he::flux_kernel<double><<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
        h->t64, static_cast<const double2 *>(psi), static_cast<double2 *>(frame), ns, lo, width,
        static_cast<const double2 *>(J), static_cast<const double2 *>(JP), field[0], field[1], field[2]);
    HE_CUDA_TRY(cudaGetLastError());
    return HE_OK;
}
