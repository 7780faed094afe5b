// Krylov workspace shared by the Arnoldi exponential and GMRES (krylov.cu, gmres.cu).
#pragma once
#include <algorithm>

#include "common.cuh"

namespace he {

// Device-resident status of one Krylov solve; kernels read `done` and return early
// once the solve has finished, so a host loop (or a captured graph) may run ahead.
struct KrylovStatus {
    int done;        // 1 once converged, broken down or failed
    int converged;   // 1 if the tolerance was met (or happy breakdown)
    int happy;       // happy breakdown seen
    int m;           // dimension of the accepted solution
    int failed;      // 1 if maxdim was reached without convergence
    int pad[3];
    double beta;     // norm of the start vector
    double estimate; // error estimate (Arnoldi) or residual estimate (GMRES)
    double hnext;    // last subdiagonal h_{j+1,j}
    double pad2;
};

constexpr int KRYLOV_BLOCKS = 296;    // 2 CTAs per SM on 148 SMs
constexpr int KRYLOV_THREADS = 256;
constexpr int KRYLOV_TILE = 8;        // basis vectors per register tile
constexpr int KRYLOV_MAXDIM = 64;
constexpr int KRYLOV_FUSED = 16;      // CGS2 with a fused update + projection sweep up to this many vectors
constexpr int KRYLOV_CAPTURE_RETRIES = 3;   // failed graph captures in a row before a workspace stops capturing

}  // namespace he

struct he_gmres_buffers;                          // gmres.cu: buffers of the device GMRES driver
void he_gmres_buffers_free(he_gmres_buffers *b);

struct he_krylov {
    int device = 0;
    size_t n = 0;                 // vector length (complex elements) of one instance
    int maxdim = 0;
    int flexible = 0;
    int count = 1;                // instances solved together (batched Arnoldi); every array below has
                                  // one slice per instance
    double2 *Q = nullptr;         // (maxdim+1) vectors; vector j of instance b at Q + (j*count + b)*n
    double2 *Z = nullptr;         // flexible GMRES: preconditioned directions (maxdim vectors)
    double2 *H = nullptr;         // (maxdim+1) x maxdim Hessenberg, column major, ld = maxdim+1
    double2 *partial = nullptr;   // KRYLOV_BLOCKS x (maxdim+1) block partial sums (scratch)
    double2 *z = nullptr;         // (maxdim+1) projections of the current CGS round
    double2 *coef = nullptr;      // maxdim combination coefficients
    double2 *work = nullptr;      // 8 * maxdim^2 complex: small dense scratch (expm / least squares)
    double *norm_partial = nullptr;   // KRYLOV_BLOCKS
    float2 *s32[2] = {nullptr, nullptr};   // complex64 operand/result of mixed-precision applies
    unsigned int *ticket = nullptr;          // device, count entries: last-block counters (0 between kernels)
    he::KrylovStatus *status = nullptr;      // device, count entries
    he::KrylovStatus *host_status = nullptr; // pinned host mirror
    size_t qs() const { return (size_t)count * n; }              // distance between basis vectors
    int blocks = he::KRYLOV_BLOCKS;   // CTAs per instance of the vector kernels (set at creation)
    bool graphs = false;              // he_krylov_set_graphs: replay repeated solves as one CUDA graph
    long long graph_key = 0;          // configuration of the last solve (0: none)
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    long long hint_key = 0;           // configuration the dimension hint belongs to
    int dim_seen = 0;                 // largest converged dimension of solves with that configuration
    int capture_fallbacks = 0;        // solves whose capture failed and were enqueued directly
    int capture_failures_in_row = 0;
    he_gmres_buffers *gmres = nullptr;  // device GMRES buffers (gmres.cu), created on first use
    int kb() const { return blocks; }
    size_t hs() const { return (size_t)(maxdim + 1) * maxdim; }  // Hessenberg size per instance
    size_t ws() const { return (size_t)8 * (maxdim + 1) * (maxdim + 1); }   // dense scratch per instance
    ~he_krylov();
};

namespace he {
// CGS2 of v against the first kc basis vectors: H column += projections, h = ||v|| into
// *hsub and the status word (skipped once the status says done).
int krylov_cgs2(he_krylov *k, int kc, double2 *v, double2 *hcol, double2 *hsub, cudaStream_t s, double happy_below);
int krylov_cgs2_fused(he_krylov *k, int kc, double2 *v, int j, cudaStream_t s, double happy_below);
int krylov_next(he_krylov *k, int kc, double2 *v, cudaStream_t s);
}  // namespace he
