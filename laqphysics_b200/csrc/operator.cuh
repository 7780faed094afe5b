// Host-side state behind an he_handle.
#pragma once
#include <string>
#include <vector>

#include "common.cuh"
#include "hpsi_kinetic.cuh"
#include "hpsi_tiled.cuh"

struct he_operator {
    int device = 0;
    int n = 0, nc = 0, nt = 0, nv = 0, nd = 0, nlam = 0;
    bool separable = false;
    bool has32 = false;
    bool tiled = false;                 // tiled kernels usable (plan built)
    int path = 1;                       // 1: tiled when possible, 0: generic gather kernel
    he::DeviceTables<double> t64{};
    he::DeviceTables<float> t32{};
    he::TiledPlan<double> p64{};
    he::TiledPlan<float> p32{};
    he::KineticPlan<double> k64{};      // kinetic-kernel plan (ntr == 0: not usable)
    he::KineticPlan<float> k32{};
    he::BandPlan<double> b64{};         // banded FP64 tensor-core kinetic plan (ntr == 0: not usable)
    he::BandPlan<float> b32{};          // the same for complex64 storage
    int *kerr = nullptr;                // device error word of the kinetic kernel
    struct TensorMapEntry {             // encoded TMA maps of recently used psi buffers
        const void *base = nullptr;
        int kind = -1;                  // 0 banded (complex128), 1 kinetic complex128, 2 kinetic complex64
        CUtensorMap map;
    };
    TensorMapEntry tmaps[16];
    int tmap_next = 0;
    double2 *coef64 = nullptr;          // field-contracted dipole coefficients (nd)
    float2 *coef32 = nullptr;
    double2 *w64[2] = {nullptr, nullptr};   // velocity gauge B-stencil scratch (n*n*nc each)
    float2 *w32[2] = {nullptr, nullptr};
    int wcap64 = 0, wcap32 = 0;         // instances the velocity-gauge scratch holds
    const double2 *tdiag = nullptr;     // diagonal of the kinetic CSR (n entries)
    he_plan_host plan;
    int mixpath = 1;                    // 1: generated (NVRTC) mixing kernel when it compiles, 0: table-driven kernel
    std::string mix_src;                // source of the generated mixing kernel (without entry points)
    int mix_state[4] = {0, 0, 0, 0};    // per variant: 0 not compiled yet, 1 ready, -1 failed (table-driven)
    void *mix_kern[4] = {nullptr, nullptr, nullptr, nullptr};   // compiled kernels (cudaKernel_t)
    int band_stages[2] = {1, 2};        // hpsi_band_kernel, length gauge, per precision (complex128,
                                        // complex64): 1 TMA stage with the registers of two CTAs per SM,
                                        // or 2 stages (he_set_band_stages; defaults = the faster on B200)
    int mix_blocks[2] = {2, 4};         // generated mixing kernel: CTAs of 128 threads per SM the register
                                        // budget is sized for (complex128, complex64)
    struct MixedGaugeTables {           // he_set_mixed_gauge (device, complex128; freed with the handle)
        bool ready = false;
        double2 *q = nullptr, *qr2h = nullptr, *F = nullptr, *c0 = nullptr, *c2 = nullptr, *qcoef = nullptr;
        int *qptr = nullptr, *qc = nullptr, *qe = nullptr;
        int nq = 0;
    } mg;
    std::vector<void *> allocations;    // every cudaMalloc made for this handle
    ~he_operator();
};

int he_fail(int status, const char *what, const char *file, int line);

bool he_build_plan(he_plan_host &P, int n, int nc, const int *ptr, const int *col, const double *tv, int nv,
                   const int *vptr, const int *vc, const int *vl, const double *vcoef, int nlam, int nd,
                   const int *dptr, const int *dc, const int *de, const double *r);

namespace he {
template <typename R>
int launch_hpsi_tiled(he_operator *h, const DeviceTables<R> &t, const TiledPlan<R> &pl, cplx<R> *coef, cplx<R> *w1,
                      cplx<R> *w2, const cplx<R> *psi, cplx<R> *out, const FieldBatch &fb, int velocity,
                      cplx<R> beta, cplx<R> gamma, cudaStream_t stream);
template <typename R> bool tiled_batchable(he_operator *h, const void *psi, int velocity);
bool tiled_fits(const he_plan_host &P, int nc, int nd);
template <typename R> bool kinetic_usable(const KineticPlan<R> &kp, const void *psi);
template <typename R>
int launch_kinetic(he_operator *h, const DeviceTables<R> &t, const KineticPlan<R> &kp, const cplx<R> *psi,
                   cplx<R> *out, cplx<R> *w1, cplx<R> *w2, R a2, int velocity, cudaStream_t stream);
int sm_count(int device);
int resident_ctas(const void *kernel, int threads, size_t smem);
std::string mix_source(const he_plan_host &P, bool dipole_real, int variant);
int jit_mix_prepare(he_operator *h, int variant);
template <typename R>
int launch_mix_jit(he_operator *h, const DeviceTables<R> &t, const cplx<R> *psi, cplx<R> *out, const cplx<R> *w1,
                   const cplx<R> *w2, const FieldBatch &fb, int velocity, cplx<R> beta, cplx<R> gamma,
                   cudaStream_t stream);
template <typename R> bool band_usable(const BandPlan<R> &bp, const void *psi);
template <typename R>
int launch_band(he_operator *h, const DeviceTables<R> &t, const BandPlan<R> &bp, const cplx<R> *psi, cplx<R> *out,
                cplx<R> *w1, cplx<R> *w2, const FieldBatch &fb, int velocity, cudaStream_t stream);
template <typename R> inline const BandPlan<R> &band_plan(const he_operator *h);
template <> inline const BandPlan<double> &band_plan<double>(const he_operator *h) { return h->b64; }
template <> inline const BandPlan<float> &band_plan<float>(const he_operator *h) { return h->b32; }
template <typename R> inline const KineticPlan<R> &kinetic_plan(const he_operator *h);
template <> inline const KineticPlan<double> &kinetic_plan<double>(const he_operator *h) { return h->k64; }
template <> inline const KineticPlan<float> &kinetic_plan<float>(const he_operator *h) { return h->k32; }
// he_apply_batched whose kernels return without work while *skip != 0 (skip may be null).
int apply_batched_gated(he_operator *h, int count, const void *psi, void *out, const double *fields, int velocity,
                        int precision, const int *skip, cudaStream_t stream);
// out += (direction . d) psi: the length-gauge dipole coupling of both electrons (the field
// derivative of H(field) along `direction`), complex128, one instance; skipped while *skip != 0.
int dipole_accumulate(he_operator *h, const double2 *psi, double2 *out, const double direction[3], const int *skip,
                      cudaStream_t stream);
// out = psi + i alpha (H(field) psi - e_ref psi), kernels skipped while *skip != 0.
int apply_shifted_gated(he_operator *h, const void *psi, void *out, const double *field, int velocity, double alpha_re,
                        double alpha_im, double e_ref, int precision, const int *skip, cudaStream_t stream);
// Separable preconditioner apply (separable.cu) whose kernels return at once while *gate != 0.
int separable_apply_gated(he_separable *h, const double2 *x, double2 *y, double2 alpha, double shift,
                          const int *gate, cudaStream_t s);
}  // namespace he
