// extern "C" entry points of libhelium_b200.so: operator handles, the drop-in
// host-pointer `tensor_apply`, and error reporting.
#include <algorithm>
#include <map>
#include <mutex>
#include <complex>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "hamiltonian.cuh"
#include "operator.cuh"

namespace {
thread_local char g_error[512] = "";
thread_local int g_status = HE_OK;
}  // namespace

void he_set_error(const char *what, const char *file, int line)
{
    const char *base = strrchr(file, '/');
    snprintf(g_error, sizeof(g_error), "%s (%s:%d)", what, base ? base + 1 : file, line);
}

int he_fail(int status, const char *what, const char *file, int line)
{
    he_set_error(what, file, line);
    g_status = status;
    return status;
}

extern "C" const char *he_last_error(void) { return g_error; }
extern "C" int he_last_status(void) { return g_status; }
extern "C" int he_version(void) { return 1; }

// ---------------------------------------------------------------------------------
// Table upload
// ---------------------------------------------------------------------------------
namespace {

template <typename T> int upload(he_operator *h, const T *src, size_t count, const T **dst)
{
    *dst = nullptr;
    if (count == 0) return HE_OK;
    void *p = nullptr;
    HE_CUDA_TRY(cudaMalloc(&p, count * sizeof(T)));
    h->allocations.push_back(p);
    HE_CUDA_TRY(cudaMemcpy(p, src, count * sizeof(T), cudaMemcpyHostToDevice));
    *dst = static_cast<const T *>(p);
    return HE_OK;
}

// complex128 host array -> device complex of precision R
template <typename R> int upload_c(he_operator *h, const double *src, size_t count, const cplx<R> **dst)
{
    std::vector<cplx<R>> tmp(count);
    for (size_t k = 0; k < count; ++k) tmp[k] = mk<R>((R)src[2 * k], (R)src[2 * k + 1]);
    return upload(h, tmp.data(), count, dst);
}

template <typename R> int upload_r(he_operator *h, const double *src, size_t count, const R **dst)
{
    std::vector<R> tmp(src, src + count);
    return upload(h, tmp.data(), count, dst);
}

int check_csr(const int *ptr, int rows, const int *col, int nnz, int ncol, const char *name)
{
    if (ptr[0] != 0 || ptr[rows] != nnz) return he_fail(HE_ERR_SHAPE, name, __FILE__, __LINE__);
    for (int i = 0; i < rows; ++i)
        if (ptr[i + 1] < ptr[i]) return he_fail(HE_ERR_SHAPE, name, __FILE__, __LINE__);
    for (int k = 0; k < nnz; ++k)
        if (col[k] < 0 || col[k] >= ncol) return he_fail(HE_ERR_SHAPE, name, __FILE__, __LINE__);
    return HE_OK;
}

template <typename R>
int build_tables(he_operator *h, he::DeviceTables<R> *t, const int *ptr, const int *col, const double *tv,
                 const double *diag, const double *d1, const double *d2, const int *vptr, const int *vc,
                 const int *vl, const double *vcoef, const double *rad, const int *dptr, const int *dc,
                 const int *de, const double *dcoef, const double *ldiff, const double *r,
                 const double *hinv)
{
    const size_t n = h->n, nc = h->nc;
    t->n = h->n; t->nc = h->nc; t->nt = h->nt; t->nv = h->nv; t->nd = h->nd; t->nlam = h->nlam;
    t->diag_separable = h->separable;
    int s;
    if ((s = upload(h, ptr, n + 1, &t->ptr))) return s;
    if ((s = upload(h, col, (size_t)h->nt, &t->col))) return s;
    if ((s = upload_c<R>(h, tv, (size_t)h->nt, &t->tv))) return s;
    t->diag = nullptr; t->d1 = nullptr; t->d2 = nullptr;
    if (h->separable) {
        if ((s = upload_c<R>(h, d1, n * nc, &t->d1))) return s;
        if ((s = upload_c<R>(h, d2, n * nc, &t->d2))) return s;
    } else {
        if ((s = upload_c<R>(h, diag, n * n * nc, &t->diag))) return s;
    }
    if ((s = upload(h, vptr, nc + 1, &t->vptr))) return s;
    if ((s = upload(h, vc, (size_t)h->nv, &t->vc))) return s;
    if ((s = upload(h, vl, (size_t)h->nv, &t->vl))) return s;
    if ((s = upload_c<R>(h, vcoef, (size_t)h->nv, &t->vcoef))) return s;
    if ((s = upload_c<R>(h, rad, n * n * (size_t)h->nlam, &t->rad))) return s;
    if ((s = upload(h, dptr, nc + 1, &t->dptr))) return s;
    if ((s = upload(h, dc, (size_t)h->nd, &t->dc))) return s;
    if ((s = upload(h, de, (size_t)h->nd, &t->de))) return s;
    if ((s = upload_c<R>(h, dcoef, 3 * (size_t)h->nd, &t->dcoef))) return s;
    if ((s = upload_r<R>(h, ldiff, (size_t)h->nd, &t->ldiff))) return s;
    if ((s = upload_c<R>(h, r, n, &t->r))) return s;
    if ((s = upload_c<R>(h, hinv, n, &t->hinv))) return s;
    return HE_OK;
}

// Kinetic (TMA-staged, FP32/FP64 FMA) plan; shares the element tables of the tiled plan.
template <typename R> int upload_kinetic(he_operator *h, const he::TiledPlan<R> *pl, he::KineticPlan<R> *kp)
{
    const he_plan_host &P = h->plan;
    int s;
    he::KineticPlan<R> k{};
    k.n = h->n; k.nc = h->nc; k.ne = P.ne; k.ntr = P.ntr; k.nct = P.nct;
    k.box_r = sizeof(R) == 8 ? P.kbox_r64 : P.kbox_r32;
    k.box_c = P.kbox_c;
    const size_t box = (size_t)k.box_r * k.box_c * sizeof(cplx<R>);
    k.stage_bytes = (int)((box + he::KIN_STAGE_ALIGN - 1) / he::KIN_STAGE_ALIGN * he::KIN_STAGE_ALIGN);
    k.estart = pl->estart; k.ereal = pl->ereal;
    if ((s = upload(h, P.koff.data(), P.koff.size(), &k.koff))) return s;
    if ((s = upload(h, P.nodeelem.data(), P.nodeelem.size(), &k.nodeelem))) return s;
    if ((s = upload_r<R>(h, P.tre.data(), P.tre.size(), &k.tre))) return s;
    if ((s = upload_r<R>(h, P.tim.data(), P.tim.size(), &k.tim))) return s;
    if ((s = upload_r<R>(h, P.bre.data(), P.bre.size(), &k.bre))) return s;
    if ((s = upload_r<R>(h, P.bim.data(), P.bim.size(), &k.bim))) return s;
    if ((s = upload(h, P.krow.data(), P.krow.size(), &k.krow))) return s;
    if ((s = upload(h, P.krbase.data(), P.krbase.size(), &k.krbase))) return s;
    if ((s = upload(h, P.krcplx.data(), P.krcplx.size(), &k.krcplx))) return s;
    if ((s = upload(h, P.kslot.data(), P.kslot.size(), &k.kslot))) return s;
    if ((s = upload(h, P.kcbase.data(), P.kcbase.size(), &k.kcbase))) return s;
    k.err = h->kerr;
    *kp = k;
    return HE_OK;
}

// Upload the tiled plan in precision R.
template <typename R> int upload_plan(he_operator *h, he::TiledPlan<R> *pl, cplx<R> **coef)
{
    const he_plan_host &P = h->plan;
    pl->n = h->n; pl->nc = h->nc; pl->ne = P.ne; pl->ntile = P.ntile;
    pl->ng = P.ng; pl->nlam = P.nlam; pl->nwd = (int)P.dwsrc.size(); pl->nwide = (int)P.wsrc.size();
    int s;
    if ((s = upload(h, P.estart.data(), P.estart.size(), &pl->estart))) return s;
    if ((s = upload(h, P.tstart.data(), P.tstart.size(), &pl->tstart))) return s;
    if ((s = upload(h, P.eoff.data(), P.eoff.size(), &pl->eoff))) return s;
    if ((s = upload(h, P.ereal.data(), P.ereal.size(), &pl->ereal))) return s;
    if ((s = upload_c<R>(h, P.blocks.data(), P.blocks.size() / 2, &pl->blocks))) return s;
    if ((s = upload_c<R>(h, P.bblocks.data(), P.bblocks.size() / 2, &pl->bblocks))) return s;
    if ((s = upload(h, P.gch.data(), P.gch.size(), &pl->gch))) return s;
    if ((s = upload(h, P.wptr.data(), P.wptr.size(), &pl->wptr))) return s;
    const int dummy_i = 0;
    const double dummy_d = 0.0;
    if ((s = upload(h, P.wsrc.empty() ? &dummy_i : P.wsrc.data(), std::max<size_t>(1, P.wsrc.size()), &pl->wsrc))) return s;
    if ((s = upload_r<R>(h, P.wcoef.empty() ? &dummy_d : P.wcoef.data(), std::max<size_t>(1, P.wcoef.size()), &pl->wcoef))) return s;
    if ((s = upload(h, P.dwptr.data(), P.dwptr.size(), &pl->dwptr))) return s;
    if ((s = upload(h, P.dwsrc.empty() ? &dummy_i : P.dwsrc.data(), std::max<size_t>(1, P.dwsrc.size()), &pl->dwsrc))) return s;
    if ((s = upload(h, P.dwel.empty() ? &dummy_i : P.dwel.data(), std::max<size_t>(1, P.dwel.size()), &pl->dwel))) return s;
    if ((s = upload(h, P.dwedge.empty() ? &dummy_i : P.dwedge.data(), std::max<size_t>(1, P.dwedge.size()), &pl->dwedge))) return s;
    void *c = nullptr;
    HE_CUDA_TRY(cudaMalloc(&c, std::max(1, h->nd) * sizeof(cplx<R>)));
    h->allocations.push_back(c);
    *coef = static_cast<cplx<R> *>(c);
    // kinetic kernel: shares the element tables of the tiled plan
    he::KineticPlan<R> *kp;
    if constexpr (sizeof(R) == 8) kp = &h->k64; else kp = &h->k32;
    *kp = he::KineticPlan<R>{};
    if (!h->kerr) {
        void *e = nullptr;
        HE_CUDA_TRY(cudaMalloc(&e, sizeof(int)));
        h->allocations.push_back(e);
        HE_CUDA_TRY(cudaMemset(e, 0, sizeof(int)));
        h->kerr = static_cast<int *>(e);
    }
    if (P.kin_ok && (s = upload_kinetic<R>(h, pl, kp))) return s;
    {   // banded tensor-core kinetic plan (FP64 fragments shared by both storage precisions)
        he::BandPlan<R> *bpp;
        if constexpr (sizeof(R) == 8) bpp = &h->b64; else bpp = &h->b32;
        *bpp = he::BandPlan<R>{};
        if (P.band_ok) {
            he::BandPlan<R> b{};
            b.n = h->n; b.nc = h->nc; b.ngroup = P.ngroup; b.ntr = P.bntr; b.nct = P.bnct;
            b.box_r = sizeof(R) == 8 ? P.bbox_r64 : P.bbox_r32;
            b.box_c = P.bbox_c;
            const size_t bytes = (size_t)b.box_r * b.box_c * sizeof(cplx<R>);
            b.stage_bytes = (int)((bytes + he::KIN_STAGE_ALIGN - 1) / he::KIN_STAGE_ALIGN * he::KIN_STAGE_ALIGN);
            if constexpr (sizeof(R) == 4) {   // the fragment and index tables of the complex128 plan are reused
                b.glo = h->b64.glo; b.gks = h->b64.gks; b.greal = h->b64.greal; b.brbase = h->b64.brbase;
                b.bcbase = h->b64.bcbase; b.frag = h->b64.frag; b.fragb = h->b64.fragb;
            } else {
                if ((s = upload(h, P.glo.data(), P.glo.size(), &b.glo))) return s;
                if ((s = upload(h, P.gks.data(), P.gks.size(), &b.gks))) return s;
                if ((s = upload(h, P.greal.data(), P.greal.size(), &b.greal))) return s;
                if ((s = upload(h, P.brbase.data(), P.brbase.size(), &b.brbase))) return s;
                if ((s = upload(h, P.bcbase.data(), P.bcbase.size(), &b.bcbase))) return s;
                if ((s = upload_c<double>(h, P.gfrag.data(), P.gfrag.size() / 2, &b.frag))) return s;
                if ((s = upload_c<double>(h, P.gfragb.data(), P.gfragb.size() / 2, &b.fragb))) return s;
            }
            b.err = h->kerr;
            if (sizeof(R) == 8 || h->b64.ntr > 0) *bpp = b;
        }
    }
    return HE_OK;
}

// Velocity-gauge scratch (two n*n*nc vectors), allocated on first use.
// Velocity-gauge scratch (two vectors of `count` instances each), grown on demand.
template <typename R> int velocity_scratch(he_operator *h, cplx<R> **w, int count)
{
    int &cap = sizeof(R) == 8 ? h->wcap64 : h->wcap32;
    if (w[0] && cap >= count) return HE_OK;
    const size_t bytes = (size_t)h->n * h->n * h->nc * sizeof(cplx<R>) * count;
    for (int k = 0; k < 2; ++k) {
        if (w[k]) {   // cudaFree waits for the device, so no kernel still reads the old buffer
            HE_CUDA_TRY(cudaFree(w[k]));
            h->allocations.erase(std::find(h->allocations.begin(), h->allocations.end(), (void *)w[k]));
            w[k] = nullptr;
        }
        void *p = nullptr;
        HE_CUDA_TRY(cudaMalloc(&p, bytes));
        h->allocations.push_back(p);
        w[k] = static_cast<cplx<R> *>(p);
    }
    cap = count;
    return HE_OK;
}

}  // namespace

he_operator::~he_operator()
{
    for (void *p : allocations) cudaFree(p);
}

cudaError_t he_smem_limit(const void *kernel, size_t bytes)
{
    static std::mutex mutex;
    static std::map<std::pair<const void *, int>, size_t> raised;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mutex);
    size_t &have = raised[{kernel, device}];
    if (have >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) have = bytes;
    return e;
}

extern "C" int he_set_path(he_handle h, int tiled)
{
    if (!h) return he_fail(HE_ERR_ARG, "null handle", __FILE__, __LINE__);
    if (tiled < 0 || tiled > 3) return he_fail(HE_ERR_ARG, "path must be 0, 1, 2 or 3", __FILE__, __LINE__);
    if (tiled && !h->tiled) return he_fail(HE_ERR_UNSUPPORTED, "tables do not admit the tiled kernels", __FILE__, __LINE__);
    h->path = tiled;
    return HE_OK;
}

extern "C" int he_set_mix(he_handle h, int generated)
{
    if (!h) return he_fail(HE_ERR_ARG, "null handle", __FILE__, __LINE__);
    if (generated != 0 && generated != 1) return he_fail(HE_ERR_ARG, "mix mode must be 0 or 1", __FILE__, __LINE__);
    h->mixpath = generated;
    return HE_OK;
}

extern "C" int he_set_mix_blocks(he_handle h, int precision, int blocks)
{
    if (!h) return he_fail(HE_ERR_ARG, "null handle", __FILE__, __LINE__);
    if (precision != HE_C128 && precision != HE_C64)
        return he_fail(HE_ERR_ARG, "precision must be HE_C128 or HE_C64", __FILE__, __LINE__);
    if (blocks < 1 || blocks > 8) return he_fail(HE_ERR_ARG, "blocks per SM must be in [1, 8]", __FILE__, __LINE__);
    const int p = precision == HE_C128 ? 0 : 1;
    if (h->mix_blocks[p] != blocks) {
        h->mix_blocks[p] = blocks;
        for (int v = 2 * p; v < 2 * p + 2; ++v) {   // recompiled (or found in the cache) on the next apply
            h->mix_state[v] = 0;
            h->mix_kern[v] = nullptr;
        }
    }
    return HE_OK;
}

extern "C" int he_set_band_stages(he_handle h, int precision, int stages)
{
    if (!h) return he_fail(HE_ERR_ARG, "null handle", __FILE__, __LINE__);
    if (precision != HE_C128 && precision != HE_C64)
        return he_fail(HE_ERR_ARG, "precision must be HE_C128 or HE_C64", __FILE__, __LINE__);
    if (stages != 1 && stages != 2) return he_fail(HE_ERR_ARG, "band kernel stages must be 1 or 2", __FILE__, __LINE__);
    h->band_stages[precision == HE_C128 ? 0 : 1] = stages;
    return HE_OK;
}

extern "C" int he_mix_status(he_handle h)
{
    if (!h) return he_fail(HE_ERR_ARG, "null handle", __FILE__, __LINE__);
    int any = 0;
    for (int v = 0; v < 4; ++v) {
        if (h->mix_state[v] < 0) return -1;
        if (h->mix_state[v] > 0) any = 1;
    }
    return any;
}

extern "C" int he_device_status(he_handle h)
{
    if (!h) return he_fail(HE_ERR_ARG, "null handle", __FILE__, __LINE__);
    if (!h->kerr) return HE_OK;
    int v = 0;
    HE_CUDA_TRY(cudaDeviceSynchronize());
    HE_CUDA_TRY(cudaMemcpy(&v, h->kerr, sizeof(int), cudaMemcpyDeviceToHost));
    if (!v) return HE_OK;
    HE_CUDA_TRY(cudaMemset(h->kerr, 0, sizeof(int)));
    return he_fail(HE_ERR_DEVICE, "a staged tile of the kinetic kernel did not arrive within its wait limit",
                   __FILE__, __LINE__);
}

extern "C" int he_create(he_handle *out, int n, int nc, int nt, const int *ptr, const int *col, const double *tv,
                         const double *diag, const double *d1, const double *d2, int nv, const int *vptr,
                         const int *vc, const int *vl, const double *vcoef, const double *rad, int nlam, int nd,
                         const int *dptr, const int *dc, const int *de, const double *dcoef, const double *ldiff,
                         const double *r, int flags)
{
    g_status = HE_OK;
    if (!out) return he_fail(HE_ERR_ARG, "null handle pointer", __FILE__, __LINE__);
    *out = nullptr;
    if (n < 1 || nc < 1 || nt < 0 || nv < 0 || nd < 0 || nlam < 1)
        return he_fail(HE_ERR_ARG, "sizes must be positive", __FILE__, __LINE__);
    if (!ptr || (nt && (!col || !tv)) || !vptr || (nv && (!vc || !vl || !vcoef)) || !rad || !dptr ||
        (nd && (!dc || !de || !dcoef || !ldiff)) || !r)
        return he_fail(HE_ERR_ARG, "null table pointer", __FILE__, __LINE__);
    const bool separable = d1 && d2;
    if (!separable && !diag) return he_fail(HE_ERR_ARG, "need diag or (d1, d2)", __FILE__, __LINE__);
    int s;
    if ((s = check_csr(ptr, n, col, nt, n, "kinetic CSR inconsistent"))) return s;
    if ((s = check_csr(vptr, nc, vc, nv, nc, "Coulomb edge list inconsistent"))) return s;
    if ((s = check_csr(dptr, nc, dc, nd, nc, "dipole edge list inconsistent"))) return s;
    for (int k = 0; k < nv; ++k)
        if (vl[k] < 0 || vl[k] >= nlam) return he_fail(HE_ERR_SHAPE, "multipole order outside rad table", __FILE__, __LINE__);
    for (int k = 0; k < nd; ++k)
        if (de[k] != 1 && de[k] != 2) return he_fail(HE_ERR_SHAPE, "dipole electron must be 1 or 2", __FILE__, __LINE__);
    for (int i = 0; i < n; ++i)
        if (r[2 * i] == 0.0 && r[2 * i + 1] == 0.0) return he_fail(HE_ERR_SHAPE, "radial node at r=0", __FILE__, __LINE__);

    he_operator *h = new he_operator();
    h->n = n; h->nc = nc; h->nt = nt; h->nv = nv; h->nd = nd; h->nlam = nlam;
    h->separable = separable;
    h->has32 = (flags & 1) != 0;
    HE_CUDA_TRY(cudaGetDevice(&h->device));
    if ((s = he_noalloc_prepare_device())) { delete h; g_status = s; return s; }
    std::vector<double> hinv(2 * (size_t)n), tdiag(2 * (size_t)n, 0.0);
    for (int i = 0; i < n; ++i) {
        const std::complex<double> v = 1.0 / (2.0 * std::complex<double>(r[2 * i], r[2 * i + 1]));
        hinv[2 * i] = v.real(); hinv[2 * i + 1] = v.imag();
        for (int k = ptr[i]; k < ptr[i + 1]; ++k)
            if (col[k] == i) { tdiag[2 * i] += tv[2 * k]; tdiag[2 * i + 1] += tv[2 * k + 1]; }
    }
    s = build_tables<double>(h, &h->t64, ptr, col, tv, diag, d1, d2, vptr, vc, vl, vcoef, rad, dptr, dc, de, dcoef,
                             ldiff, r, hinv.data());
    if (!s && h->has32)
        s = build_tables<float>(h, &h->t32, ptr, col, tv, diag, d1, d2, vptr, vc, vl, vcoef, rad, dptr, dc, de,
                                dcoef, ldiff, r, hinv.data());
    if (!s) {
        const double2 *td = nullptr;
        s = upload_c<double>(h, tdiag.data(), (size_t)n, &td);
        h->tdiag = td;
    }
    if (!s && he_build_plan(h->plan, n, nc, ptr, col, tv, nv, vptr, vc, vl, vcoef, nlam, nd, dptr, dc, de, r) &&
        he::tiled_fits(h->plan, nc, nd)) {
        s = upload_plan<double>(h, &h->p64, &h->coef64);
        if (!s && h->has32) s = upload_plan<float>(h, &h->p32, &h->coef32);
        h->tiled = !s;
        bool dipole_real = true;
        for (long long k = 0; k < 3LL * nd; ++k) dipole_real = dipole_real && dcoef[2 * k + 1] == 0.0;
        h->mix_src = he::mix_source(h->plan, dipole_real, -2);
    }
    if (s) { delete h; g_status = s; return s; }
    *out = h;
    return HE_OK;
}

extern "C" int he_destroy(he_handle h)
{
    delete h;
    return HE_OK;
}

extern "C" int he_info(he_handle h, long long *values, int count)
{
    if (!h || !values) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    const long long all[] = {h->n, h->nc, h->nt, h->nv, h->nd, h->nlam, h->separable, h->has32, h->device,
                             h->tiled, h->path, h->plan.ne, h->plan.ntile, h->plan.ng,
                             (long long)h->plan.wsrc.size(), (long long)h->plan.dwsrc.size(),
                             h->b64.ntr > 0, h->k64.ntr > 0};
    for (int k = 0; k < count && k < (int)(sizeof(all) / sizeof(all[0])); ++k) values[k] = all[k];
    return HE_OK;
}

namespace {
int apply_common(he_handle h, const void *psi, void *out, const he::FieldBatch &fb, int velocity, int precision,
                 double beta_re, double beta_im, double gamma_re, double gamma_im, void *stream)
{
    g_status = HE_OK;
    if (!h || !psi || !out) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (velocity != 0 && velocity != 1) return he_fail(HE_ERR_ARG, "velocity must be 0 or 1", __FILE__, __LINE__);
    if (psi == out) return he_fail(HE_ERR_ARG, "H·psi cannot run in place", __FILE__, __LINE__);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t N = (size_t)h->n * h->n * h->nc;
    int s = HE_OK;
    const bool tiled = h->tiled && h->path >= 1;
    if (precision == HE_C128) {
        const double2 beta = mk<double>(beta_re, beta_im), gamma = mk<double>(gamma_re, gamma_im);
        const double2 *x = static_cast<const double2 *>(psi);
        double2 *y = static_cast<double2 *>(out);
        if (velocity && tiled && (s = velocity_scratch<double>(h, h->w64, fb.count))) return g_status = s;
        if (tiled && (fb.count == 1 || he::tiled_batchable<double>(h, psi, velocity))) {
            s = he::launch_hpsi_tiled<double>(h, h->t64, h->p64, h->coef64, h->w64[0], h->w64[1], x, y, fb, velocity,
                                              beta, gamma, st);
        } else {
            for (int b = 0; b < fb.count && !s; ++b) {   // one instance at a time
                he::FieldBatch one{1, {}, fb.skip};
                for (int a = 0; a < 3; ++a) one.f[0][a] = fb.f[b][a];
                s = tiled ? he::launch_hpsi_tiled<double>(h, h->t64, h->p64, h->coef64, h->w64[0], h->w64[1],
                                                          x + b * N, y + b * N, one, velocity, beta, gamma, st)
                          : he::launch_hpsi<double>(h->t64, x + b * N, y + b * N, one.f[0], velocity, beta, gamma, st);
            }
        }
    } else if (precision == HE_C64) {
        if (!h->has32) return he_fail(HE_ERR_UNSUPPORTED, "handle built without complex64 tables", __FILE__, __LINE__);
        const float2 beta = mk<float>((float)beta_re, (float)beta_im), gamma = mk<float>((float)gamma_re, (float)gamma_im);
        const float2 *x = static_cast<const float2 *>(psi);
        float2 *y = static_cast<float2 *>(out);
        if (velocity && tiled && (s = velocity_scratch<float>(h, h->w32, fb.count))) return g_status = s;
        if (tiled && (fb.count == 1 || he::tiled_batchable<float>(h, psi, velocity))) {
            s = he::launch_hpsi_tiled<float>(h, h->t32, h->p32, h->coef32, h->w32[0], h->w32[1], x, y, fb, velocity,
                                             beta, gamma, st);
        } else {
            for (int b = 0; b < fb.count && !s; ++b) {
                he::FieldBatch one{1, {}, fb.skip};
                for (int a = 0; a < 3; ++a) one.f[0][a] = fb.f[b][a];
                s = tiled ? he::launch_hpsi_tiled<float>(h, h->t32, h->p32, h->coef32, h->w32[0], h->w32[1],
                                                         x + b * N, y + b * N, one, velocity, beta, gamma, st)
                          : he::launch_hpsi<float>(h->t32, x + b * N, y + b * N, one.f[0], velocity, beta, gamma, st);
            }
        }
    } else {
        return he_fail(HE_ERR_ARG, "precision must be HE_C128 or HE_C64", __FILE__, __LINE__);
    }
    g_status = s;
    return s;
}

he::FieldBatch single_field(const double *field)
{
    he::FieldBatch fb{1, {}};
    for (int a = 0; a < 3; ++a) fb.f[0][a] = field[a];
    return fb;
}
}  // namespace

extern "C" int he_apply(he_handle h, const void *psi, void *out, const double *field, int velocity, int precision,
                        void *stream)
{
    if (!field) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    return apply_common(h, psi, out, single_field(field), velocity, precision, 0.0, 0.0, 1.0, 0.0, stream);
}

namespace he {
int apply_batched_gated(he_handle h, int count, const void *psi, void *out, const double *fields, int velocity,
                        int precision, const int *skip, cudaStream_t stream)
{
    if (!fields) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    if (count < 1 || count > he::HE_BATCH_MAX)
        return he_fail(HE_ERR_ARG, "batch count must be between 1 and 64", __FILE__, __LINE__);
    he::FieldBatch fb{count, {}, skip};
    for (int b = 0; b < count; ++b)
        for (int a = 0; a < 3; ++a) fb.f[b][a] = fields[3 * b + a];
    return apply_common(h, psi, out, fb, velocity, precision, 0.0, 0.0, 1.0, 0.0, stream);
}
}  // namespace he

extern "C" int he_apply_batched(he_handle h, int count, const void *psi, void *out, const double *fields, int velocity,
                                int precision, void *stream)
{
    return he::apply_batched_gated(h, count, psi, out, fields, velocity, precision, nullptr,
                                   static_cast<cudaStream_t>(stream));
}

namespace he {
int apply_shifted_gated(he_handle h, const void *psi, void *out, const double *field, int velocity, double alpha_re,
                        double alpha_im, double e_ref, int precision, const int *skip, cudaStream_t stream)
{
    const double ga_re = -alpha_im, ga_im = alpha_re;     // i*alpha
    if (!field) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    he::FieldBatch fb = single_field(field);
    fb.skip = skip;
    return apply_common(h, psi, out, fb, velocity, precision, 1.0 - ga_re * e_ref, -ga_im * e_ref, ga_re, ga_im,
                        stream);
}
}  // namespace he

extern "C" int he_apply_shifted(he_handle h, const void *psi, void *out, const double *field, int velocity,
                                double alpha_re, double alpha_im, double e_ref, int precision, void *stream)
{
    // psi + i alpha (H psi - e_ref psi) = (1 - i alpha e_ref) psi + (i alpha) H psi
    const double ga_re = -alpha_im, ga_im = alpha_re;     // i*alpha
    if (!field) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    return apply_common(h, psi, out, single_field(field), velocity, precision, 1.0 - ga_re * e_ref, -ga_im * e_ref, ga_re, ga_im,
                        stream);
}

extern "C" int he_diagonal(he_handle h, void *out, void *stream)
{
    g_status = HE_OK;
    if (!h || !out) return he_fail(HE_ERR_ARG, "null argument", __FILE__, __LINE__);
    return g_status = he::launch_diagonal(h->t64, h->tdiag, static_cast<double2 *>(out), static_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------------
// Drop-in host-pointer tensor_apply (src/kernels.f90:119-127 signature).
// ---------------------------------------------------------------------------------
extern "C" void tensor_apply(int n, int nc, int nt, const int *ptr, const int *col, const double *tv,
                             const double *diag, int nv, const int *vptr, const int *vc, const int *vl,
                             const double *vcoef, const double *rad, int nd, const int *dptr, const int *dc,
                             const int *de, const double *dcoef, const double *ldiff, const double *r,
                             const double *field, int velocity, const double *psi, double *out)
{
    g_status = HE_OK;
    if (!psi || !out || !field || n < 1 || nc < 1) { he_fail(HE_ERR_ARG, "bad tensor_apply argument", __FILE__, __LINE__); return; }
    int nlam = 1;
    for (int k = 0; k < nv; ++k) nlam = std::max(nlam, vl[k] + 1);
    he_handle h = nullptr;
    if (he_create(&h, n, nc, nt, ptr, col, tv, diag, nullptr, nullptr, nv, vptr, vc, vl, vcoef, rad, nlam, nd, dptr,
                  dc, de, dcoef, ldiff, r, 0) != HE_OK)
        return;
    const size_t bytes = (size_t)n * n * nc * 2 * sizeof(double);
    void *dpsi = nullptr, *dout = nullptr;
    cudaError_t e = cudaMalloc(&dpsi, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&dout, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(dpsi, psi, bytes, cudaMemcpyHostToDevice);
    int s = HE_ERR_CUDA;
    if (e == cudaSuccess) s = he_apply(h, dpsi, dout, field, velocity, HE_C128, nullptr);
    if (s == HE_OK) {
        e = cudaMemcpy(out, dout, bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) s = HE_ERR_CUDA;
    }
    if (e != cudaSuccess) he_set_error(cudaGetErrorString(e), __FILE__, __LINE__);
    cudaFree(dpsi);
    cudaFree(dout);
    he_destroy(h);
    g_status = s;
}
