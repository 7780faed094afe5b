// Norms of a batch of complex128 vectors with no device allocation.
//
// he_vec_residual_norm (vecops.cu) keeps its block partial sums in scratch that it
// cudaMalloc's on first use.  Some callers of this library cannot let a call allocate:
// a host process whose device memory is already handed to a pool allocator (an extra
// cudaMalloc can fail or fragment that pool), a latency-critical propagation loop that
// must not stall on the allocator's implicit device synchronisation, and a library
// embedded in another runtime that forbids device allocations outside its own
// allocator.  he_vec_norms_noalloc serves them: its scratch is the file-scope device
// array below, sized for NOALLOC_MAX_VECTORS vectors.
//
// When the array comes into being.  The array belongs to this file's CUDA module.  Under
// CUDA's lazy module loading (the default since CUDA 12.2) the driver loads the module,
// and allocates the array on that device, the first time the process touches it on a
// device: the address lookup below.  That lookup happens (a) in he_create, for the device
// an operator is created on, and (b) otherwise at the first he_vec_norms_noalloc call on a
// device.  A caller that hands the device's memory to a pool allocator should therefore
// create its operator, or make one he_vec_norms_noalloc call, before the pool takes the
// memory; with CUDA_MODULE_LOADING=EAGER the array is allocated when the context is
// created.  From then on the array stays allocated until the process exits and no call of
// this entry point allocates device memory.  The address lookup of (b) must not run during
// a stream capture, so that first call belongs before any capture on the device.
//
// The array is shared by all calls and keeps the last call's contents; every entry a
// call reads is written earlier in the same call, so nothing needs clearing, but calls
// that overlap on the GPU (e.g. on two streams) race on it and must be serialised by
// the caller.
#include <mutex>

#include "common.cuh"
#include "operator.cuh"

namespace {

constexpr int NOALLOC_MAX_VECTORS = 64;    // largest batch one call accepts
constexpr int NOALLOC_BLOCKS = 296;        // same reduction grid as he_vec_residual_norm
constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_MAX_DEVICES = 64;

// Block partials (NOALLOC_BLOCKS x NOALLOC_MAX_VECTORS) followed by the final norms:
// (296 + 1) x 64 doubles = 152,064 bytes per device.
static __device__ __align__(256) double g_noalloc_scratch[(NOALLOC_BLOCKS + 1) * NOALLOC_MAX_VECTORS];

std::mutex g_noalloc_mutex;
double *g_noalloc_address[NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array on the current device (looked up once per device).
int scratch_address(double **out)
{
    int dev = 0;
    HE_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return he_fail(HE_ERR_ARG, "device index out of range", __FILE__, __LINE__);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_address[dev]) {
        double *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) {
            he_set_error(cudaGetErrorString(e), __FILE__, __LINE__);
            return HE_ERR_CUDA;
        }
        g_noalloc_address[dev] = ptr;
    }
    *out = g_noalloc_address[dev];
    return HE_OK;
}

// Per-block sums of |x_v|^2 for every vector v of the batch (same thread order and
// reduction tree as vecops.cu's residual_kernel).
__global__ void __launch_bounds__(NOALLOC_THREADS)
norms_partial_kernel(size_t n, int count, const double2 *__restrict__ x, size_t ld, double *__restrict__ scratch)
{
    __shared__ double red[NOALLOC_THREADS / 32];
    for (int v = 0; v < count; ++v) {
        const double2 *xv = x + (size_t)v * ld;
        double s = 0;
        for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x)
            s += cabs2<double>(xv[p]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int w = 0; w < NOALLOC_THREADS / 32; ++w) t += red[w];
            scratch[(size_t)blockIdx.x * NOALLOC_MAX_VECTORS + v] = t;
        }
        __syncthreads();
    }
}

// norms[v] = sqrt(sum over blocks, in block order) into the last scratch row.
__global__ void norms_finish_kernel(int count, double *scratch)
{
    for (int v = threadIdx.x; v < count; v += blockDim.x) {
        double s = 0;
        for (int b = 0; b < NOALLOC_BLOCKS; ++b) s += scratch[(size_t)b * NOALLOC_MAX_VECTORS + v];
        scratch[(size_t)NOALLOC_BLOCKS * NOALLOC_MAX_VECTORS + v] = sqrt(s);
    }
}

}  // namespace

// Resolve the scratch array on the current device (loads this module there under lazy
// loading); called by he_create so an operator's device holds the array from set-up on.
int he_noalloc_prepare_device()
{
    double *unused = nullptr;
    return scratch_address(&unused);
}

// norms[v] = ||x_v|| for v < count, x_v = x + v*ld (complex128 device vectors of n
// elements); `norms` is host memory of count doubles.  Blocks the host until done.
extern "C" int he_vec_norms_noalloc(long long n, int count, const void *x, long long ld, double *norms, void *stream)
{
    if (n < 0 || !x || !norms) return he_fail(HE_ERR_ARG, "bad batched-norm argument", __FILE__, __LINE__);
    if (count < 1 || count > NOALLOC_MAX_VECTORS)
        return he_fail(HE_ERR_ARG, "he_vec_norms_noalloc: count must be between 1 and 64 (the static scratch holds 64 vectors)",
                       __FILE__, __LINE__);
    if (count > 1 && ld < n) return he_fail(HE_ERR_ARG, "leading dimension smaller than the vector length", __FILE__, __LINE__);
    double *scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    norms_partial_kernel<<<NOALLOC_BLOCKS, NOALLOC_THREADS, 0, s>>>((size_t)n, count, static_cast<const double2 *>(x),
                                                                     (size_t)ld, scratch);
    norms_finish_kernel<<<1, 64, 0, s>>>(count, scratch);
    HE_CUDA_TRY(cudaGetLastError());
    HE_CUDA_TRY(cudaMemcpyAsync(norms, scratch + (size_t)NOALLOC_BLOCKS * NOALLOC_MAX_VECTORS, count * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
    HE_CUDA_TRY(cudaStreamSynchronize(s));
    return HE_OK;
}
