// Channel mixing of H·psi as a kernel generated for the operator's own coupling
// structure and compiled with NVRTC for sm_100a when the operator is first applied.
//
// The Coulomb multipoles (src/kernels.f90:132-143: sum_lam rad(i,j,lam) sum_c' vcoef
// psi(i,j,c')) and the dipole couplings (:145-168) are the same for every point of the
// radial grid, so the generated kernel unrolls every edge with its coefficient as an
// exact literal: one thread per point (or per point and output group on small grids), the group's output channels in registers, each
// source loaded once per block of multipoles, no coefficient loads and no padded slots.
// The dipole coefficients depend on the field; each CTA contracts them once into shared
// memory (zero below 1e-30, the skip of src/kernels.f90:145).
//
// Per point and output group:
//   a_d   = (H psi)_radial[c_d]                                     (kinetic kernel output)
//   a_d  += rad_lam t_d,  t_d = sum_(s, w) w psi_s                  (per multipole lam)
//   length:   a_d += r_e   sum_k coef_k psi_(s_k)                    (per electron e)
//   velocity: a_d += 1/(2 r_e) sum_k i coef_k ldiff_k psi_(s_k) + sum_k i coef_k W_e[s_k]
//   out[c_d] = beta psi[c_d] + gamma a_d
#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <sstream>
#include <string>

#include "common.cuh"
#include "operator.cuh"

namespace he {

namespace {

const char *kPrelude = R"(// generated channel-mixing kernel
struct FieldBatch { int count; double f[HE_BATCH_MAX][3]; const int *skip; };
struct __align__(16) cd { double x, y; };
struct __align__(8) cf { float x, y; };
template <typename R> struct cx;
template <> struct cx<double> { typedef cd T; };
template <> struct cx<float> { typedef cf T; };
__device__ __forceinline__ double f3(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float f3(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <typename R> __device__ __forceinline__ typename cx<R>::T mk(R a, R b) { typename cx<R>::T z; z.x = a; z.y = b; return z; }
// c + a b
template <typename R> __device__ __forceinline__ typename cx<R>::T cfma(typename cx<R>::T a, typename cx<R>::T b, typename cx<R>::T c)
{ c.x = f3(a.x, b.x, c.x); c.x = f3(-a.y, b.y, c.x); c.y = f3(a.x, b.y, c.y); c.y = f3(a.y, b.x, c.y); return c; }
// c + s b, s real
template <typename R> __device__ __forceinline__ typename cx<R>::T rfma(R s, typename cx<R>::T b, typename cx<R>::T c)
{ c.x = f3(s, b.x, c.x); c.y = f3(s, b.y, c.y); return c; }
// c + (i s) b, s real
template <typename R> __device__ __forceinline__ typename cx<R>::T ifma(R s, typename cx<R>::T b, typename cx<R>::T c)
{ c.x = f3(-s, b.y, c.x); c.y = f3(s, b.x, c.y); return c; }
template <typename R> __device__ __forceinline__ typename cx<R>::T cmul(typename cx<R>::T a, typename cx<R>::T b)
{ return mk<R>(f3(a.x, b.x, -a.y * b.y), f3(a.x, b.y, a.y * b.x)); }
// streaming (evict-first) access to the output, read once and written once per point, so
// that L1 keeps the channels of psi and the multipoles that several groups read
__device__ __forceinline__ cd ld_stream(const cd *p)
{ cd v; asm volatile("ld.global.cs.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p)); return v; }
__device__ __forceinline__ cf ld_stream(const cf *p)
{ cf v; asm volatile("ld.global.cs.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p)); return v; }
__device__ __forceinline__ void st_stream(cd *p, cd v)
{ asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};" :: "l"(p), "d"(v.x), "d"(v.y) : "memory"); }
__device__ __forceinline__ void st_stream(cf *p, cf v)
{ asm volatile("st.global.cs.v2.f32 [%0], {%1, %2};" :: "l"(p), "f"(v.x), "f"(v.y) : "memory"); }
)";

std::string lit(double v)
{
    char buf[40];
    std::snprintf(buf, sizeof(buf), "%.17g", v);
    std::string s(buf);
    if (s.find_first_of(".eEn") == std::string::npos) s += ".0";
    return "(R)" + s;
}

}  // namespace

// CTAs of 128 threads per SM the generated kernels are compiled for (register budget):
// the complex128 groups need more registers than the complex64 ones.
constexpr int MIXJ_MIN_BLOCKS_D = 2, MIXJ_MIN_BLOCKS_F = 4;

std::string mix_entry(int v, int min_blocks);

// CUDA source of the generated kernel for a plan (variant -1: all four entry points,
// -2: none, 0..3: one).  `dipole_real`: every dcoef entry is
// real, so field-contracted coefficients are real (length) or imaginary (velocity).
std::string mix_source(const he_plan_host &P, bool dipole_real, int variant)
{
    // The groups are __noinline__ functions: each is register-allocated on its own, so the
    // loads of one group are not hoisted into another (no spills at two CTAs of 128 per SM).
    std::ostringstream o;
    o << kPrelude;
    o << "template <typename R, bool VEL>\n__device__ __forceinline__ void mix_body(\n"
         "    const typename cx<R>::T *__restrict__ psi, typename cx<R>::T *__restrict__ out,\n"
         "    const typename cx<R>::T *__restrict__ rad, const typename cx<R>::T *__restrict__ rt,\n"
         "    const typename cx<R>::T *__restrict__ w1, const typename cx<R>::T *__restrict__ w2,\n"
         "    const typename cx<R>::T *__restrict__ dcoef, const R *__restrict__ ldiff, long long nn, int n, int nd,\n"
         "    int nc, const FieldBatch &fs, typename cx<R>::T beta, typename cx<R>::T gamma)\n{\n"
         "    typedef typename cx<R>::T C;\n"
         "    if (fs.skip && *fs.skip) return;   // the solve that enqueued this apply has converged\n"
         "    // instance blockIdx.z of a batch: its own field and its block of nc channels\n"
         "    const long long shift = (long long)blockIdx.z * nc * nn;\n"
         "    psi += shift; out += shift;\n"
         "    if (VEL) { w1 += shift; w2 += shift; }\n"
         "    const R f0 = (R)fs.f[blockIdx.z][0], f1 = (R)fs.f[blockIdx.z][1], f2 = (R)fs.f[blockIdx.z][2];\n"
         "    extern __shared__ __align__(16) unsigned char smem_raw[];\n"
         "    C *K = reinterpret_cast<C *>(smem_raw), *KW = K + nd;\n"
         "    for (int k = threadIdx.x; k < nd; k += blockDim.x) {\n"
         "        C v = mk<R>(f0 * dcoef[3 * k].x, f0 * dcoef[3 * k].y);\n"
         "        v = rfma<R>(f1, dcoef[3 * k + 1], v);\n"
         "        v = rfma<R>(f2, dcoef[3 * k + 2], v);\n"
         "        if (sqrt(v.x * v.x + v.y * v.y) < (R)1e-30) v = mk<R>(0, 0);\n"
         "        const C iv = mk<R>(-v.y, v.x);\n"
         "        K[k] = VEL ? mk<R>(iv.x * ldiff[k], iv.y * ldiff[k]) : v;\n"
         "        if (VEL) KW[k] = iv;\n"
         "    }\n"
         "    __syncthreads();\n"
         "    // grid y = point blocks; grid x = 1: a thread runs every output group of its point (large\n"
         "    // grids), else x = output group (small grids; fastest axis, so one point block's groups share L2)\n"
         "    for (long long pb = blockIdx.y; pb * blockDim.x < nn; pb += gridDim.y) {\n"
         "        const long long p = pb * blockDim.x + threadIdx.x;\n"
         "        if (p >= nn) return;\n"
         "        const C re1 = rt[p % n], re2 = rt[p / n];\n"
         "        if (gridDim.x == 1) {\n";
    for (size_t g = 0; g < P.mix.size(); ++g)
        o << "            mix_group" << g << "<R, VEL>(psi, out, rad, w1, w2, K, KW, p, nn, re1, re2, beta, gamma);\n";
    o << "        } else {\n            switch (blockIdx.x) {\n";
    for (size_t g = 0; g < P.mix.size(); ++g)
        o << "            case " << g << ": mix_group" << g
          << "<R, VEL>(psi, out, rad, w1, w2, K, KW, p, nn, re1, re2, beta, gamma); break;\n";
    o << "            }\n        }\n    }\n}\n";
    const std::string body = o.str().substr(std::string(kPrelude).size());
    o.str("");
    // coefficient use: real part (length, dipole_real), imaginary part (velocity, dipole_real) or full complex
    auto dip_term = [&](const char *acc, const char *kref, const char *x) {
        std::ostringstream t;
        if (dipole_real)
            t << acc << " = VEL ? ifma<R>(" << kref << ".y, " << x << ", " << acc << ") : rfma<R>(" << kref << ".x, " << x
              << ", " << acc << ");";
        else
            t << acc << " = cfma<R>(" << kref << ", " << x << ", " << acc << ");";
        return t.str();
    };
    for (size_t g = 0; g < P.mix.size(); ++g) {
        const MixGroup &G = P.mix[g];
        o << "template <typename R, bool VEL>\n__device__ __noinline__ void mix_group" << g
          << "(const typename cx<R>::T *__restrict__ psi, typename cx<R>::T *__restrict__ out,\n"
             "    const typename cx<R>::T *__restrict__ rad, const typename cx<R>::T *__restrict__ w1,\n"
             "    const typename cx<R>::T *__restrict__ w2, const typename cx<R>::T *K, const typename cx<R>::T *KW,\n"
             "    long long p, long long nn, typename cx<R>::T re1, typename cx<R>::T re2, typename cx<R>::T beta,\n"
             "    typename cx<R>::T gamma)\n{\n"
             "    typedef typename cx<R>::T C;\n"
             "    const C Z = mk<R>(0, 0);\n";
        o << "    {   // group " << g << "\n";
        for (size_t d = 0; d < G.out.size(); ++d) o << "        C a" << d << " = ld_stream(out + p + nn * " << G.out[d] << "LL);\n";
        for (const MixBlock &B : G.blocks) {
            o << "        {\n";
            for (size_t s = 0; s < B.src.size(); ++s)
                o << "            const C x" << s << " = psi[p + nn * " << B.src[s] << "LL];\n";
            for (const MixTerm &T : B.terms) {
                std::set<int> outs(T.d.begin(), T.d.end());
                o << "            {   // multipole " << T.lam << "\n";
                o << "                const C r = rad[p + nn * " << T.lam << "LL];\n";
                for (int d : outs) o << "                C t" << d << " = Z;\n";
                for (size_t e = 0; e < T.d.size(); ++e)
                    o << "                t" << T.d[e] << " = rfma<R>(" << lit(T.w[e]) << ", x" << T.s[e] << ", t" << T.d[e]
                      << ");\n";
                for (int d : outs) o << "                a" << d << " = cfma<R>(r, t" << d << ", a" << d << ");\n";
                o << "            }\n";
            }
            o << "        }\n";
        }
        for (int e = 0; e < 2; ++e) {
            if (G.dd[e].empty()) continue;
            std::set<int> outs(G.dd[e].begin(), G.dd[e].end());
            o << "        {   // dipole, electron " << e + 1 << "\n";
            for (int d : outs) o << "            C u" << d << " = Z;\n";
            o << "            if (VEL) {\n";
            for (int d : outs) o << "                C z" << d << " = Z;\n";
            for (size_t k = 0; k < G.dd[e].size(); ++k) {
                const int d = G.dd[e][k], s = G.ds[e][k], kk = G.dk[e][k];
                o << "                { const C y = psi[p + nn * " << s << "LL]; "
                  << dip_term(("u" + std::to_string(d)).c_str(), ("K[" + std::to_string(kk) + "]").c_str(), "y")
                  << " }\n";
                o << "                { const C y = w" << e + 1 << "[p + nn * " << s << "LL]; "
                  << dip_term(("z" + std::to_string(d)).c_str(), ("KW[" + std::to_string(kk) + "]").c_str(), "y")
                  << " }\n";
            }
            for (int d : outs)
                o << "                a" << d << " = cfma<R>(re" << e + 1 << ", u" << d << ", a" << d << "); a" << d
                  << ".x += z" << d << ".x; a" << d << ".y += z" << d << ".y;\n";
            o << "            } else {\n";
            for (size_t k = 0; k < G.dd[e].size(); ++k) {
                const int d = G.dd[e][k], s = G.ds[e][k], kk = G.dk[e][k];
                o << "                { const C y = psi[p + nn * " << s << "LL]; "
                  << dip_term(("u" + std::to_string(d)).c_str(), ("K[" + std::to_string(kk) + "]").c_str(), "y")
                  << " }\n";
            }
            for (int d : outs) o << "                a" << d << " = cfma<R>(re" << e + 1 << ", u" << d << ", a" << d << ");\n";
            o << "            }\n        }\n";
        }
        for (size_t d = 0; d < G.out.size(); ++d)
            o << "        st_stream(out + p + nn * " << G.out[d] << "LL, cfma<R>(gamma, a" << d << ", cmul<R>(beta, psi[p + nn * "
              << G.out[d] << "LL])));\n";
        o << "    }\n}\n";
    }
    const std::string group_fns = o.str();
    o.str("");
    o << "#define HE_BATCH_MAX " << HE_BATCH_MAX << "\n" << kPrelude << group_fns << body;
    if (variant == -1)
        for (int v = 0; v < 4; ++v) o << mix_entry(v, 0);
    else if (variant >= 0)
        o << mix_entry(variant, 0);
    return o.str();
}

// Entry point of one variant: 0/1 complex128 length/velocity, 2/3 complex64; min_blocks
// (> 0) overrides the default CTAs per SM of the register budget.
std::string mix_entry(int v, int min_blocks)
{
    const char *names[4] = {"he_mix_d0", "he_mix_d1", "he_mix_f0", "he_mix_f1"};
    const bool dbl = v < 2, vel = v & 1;
    const char *R = dbl ? "double" : "float", *C = dbl ? "cd" : "cf";
    std::ostringstream o;
    const int blocks = min_blocks > 0 ? min_blocks : (dbl ? MIXJ_MIN_BLOCKS_D : MIXJ_MIN_BLOCKS_F);
    o << "extern \"C\" __global__ void __launch_bounds__(128, " << blocks << ") "
      << names[v] << "(const " << C << " *psi, " << C << " *out, const " << C << " *rad, const " << C << " *rt, const " << C
      << " *w1, const " << C << " *w2, const " << C << " *dcoef, const " << R
      << " *ldiff, long long nn, int n, int nd, int nc, const FieldBatch fs, " << C << " beta, " << C
      << " gamma)\n{ mix_body<" << R << ", " << (vel ? "true" : "false")
      << ">(psi, out, rad, rt, w1, w2, dcoef, ldiff, nn, n, nd, nc, fs, beta, gamma); }\n";
    return o.str();
}

// NVRTC compile of a generated source for sm_100a.  Returns the cubin, or an empty vector
// with the compiler log in `log`.
std::vector<char> nvrtc_compile(const std::string &src, std::string &log)
{
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "he_mix.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
        log = "nvrtcCreateProgram failed";
        return {};
    }
    const char *opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-lineinfo"};
    const nvrtcResult r = nvrtcCompileProgram(prog, 3, opts);
    size_t n = 0;
    nvrtcGetProgramLogSize(prog, &n);
    log.assign(n, '\0');
    if (n) nvrtcGetProgramLog(prog, &log[0]);
    std::vector<char> cubin;
    if (r == NVRTC_SUCCESS) {
        size_t m = 0;
        nvrtcGetCUBINSize(prog, &m);
        cubin.resize(m);
        nvrtcGetCUBIN(prog, cubin.data());
    }
    nvrtcDestroyProgram(&prog);
    return cubin;
}

namespace {

const char *kEntry[4] = {"he_mix_d0", "he_mix_d1", "he_mix_f0", "he_mix_f1"};

struct JitKernel {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kern = nullptr;
};

std::mutex g_jit_mutex;
std::map<std::string, std::shared_ptr<JitKernel>> g_jit_cache;   // keyed by source text

// Directory of compiled kernels: $HE_JIT_CACHE, else "jit" beside this library.
std::string cache_dir()
{
    if (const char *env = std::getenv("HE_JIT_CACHE")) return env;
    Dl_info info;
    if (dladdr(reinterpret_cast<void *>(&he_mix_status), &info) && info.dli_fname) {
        std::string path(info.dli_fname);
        const size_t slash = path.rfind('/');
        return (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/jit";
    }
    return "";
}

std::string read_file(const std::string &path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) return "";
    std::ostringstream o;
    o << f.rdbuf();
    return o.str();
}

void write_file(const std::string &path, const std::string &data)
{
    const std::string tmp = path + ".tmp" + std::to_string((long long)getpid());
    {
        std::ofstream f(tmp, std::ios::binary);
        if (!f) return;
        f.write(data.data(), (std::streamsize)data.size());
        if (!f) { std::remove(tmp.c_str()); return; }
    }
    std::rename(tmp.c_str(), path.c_str());
}

// Cubin of a source: from the on-disk cache when its stored source matches, else NVRTC
// (and stored).
std::vector<char> cubin_for(const std::string &src, std::string &log)
{
    const std::string dir = cache_dir();
    char key[32];
    std::snprintf(key, sizeof(key), "%016zx", std::hash<std::string>{}(src));
    const std::string base = dir.empty() ? "" : dir + "/mix_" + key;
    if (!base.empty() && read_file(base + ".cu") == src) {
        const std::string bin = read_file(base + ".cubin");
        if (!bin.empty()) return std::vector<char>(bin.begin(), bin.end());
    }
    std::vector<char> cubin = nvrtc_compile(src, log);
    if (!cubin.empty() && !base.empty()) {
        mkdir(dir.c_str(), 0755);
        write_file(base + ".cubin", std::string(cubin.begin(), cubin.end()));
        write_file(base + ".cu", src);
    }
    return cubin;
}

}  // namespace

// The generated kernel of one variant (0 complex128 length, 1 complex128 velocity,
// 2 complex64 length, 3 complex64 velocity), compiled and loaded on first use and shared
// by operators with the same structure.  On failure the operator falls back to the
// table-driven mixing kernel for that variant.
int jit_mix_prepare(he_operator *h, int variant)
{
    if (h->mix_state[variant] != 0) return h->mix_state[variant] > 0 ? HE_OK : HE_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_jit_mutex);
    const std::string src = h->mix_src + mix_entry(variant, h->mix_blocks[variant < 2 ? 0 : 1]);
    auto it = g_jit_cache.find(src);
    if (it == g_jit_cache.end()) {
        std::string log;
        const std::vector<char> cubin = cubin_for(src, log);
        if (cubin.empty()) {
            h->mix_state[variant] = -1;
            return he_fail(HE_ERR_UNSUPPORTED, ("generated mixing kernel did not compile: " + log.substr(0, 400)).c_str(),
                           __FILE__, __LINE__);
        }
        auto J = std::make_shared<JitKernel>();
        HE_CUDA_TRY(cudaLibraryLoadData(&J->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
        HE_CUDA_TRY(cudaLibraryGetKernel(&J->kern, J->lib, kEntry[variant]));
        it = g_jit_cache.emplace(src, J).first;
    }
    h->mix_kern[variant] = it->second->kern;
    h->mix_state[variant] = 1;
    return HE_OK;
}

template <typename R>
int launch_mix_jit(he_operator *h, const DeviceTables<R> &t, const cplx<R> *psi, cplx<R> *out, const cplx<R> *w1,
                   const cplx<R> *w2, const FieldBatch &fb, int velocity, cplx<R> beta, cplx<R> gamma,
                   cudaStream_t stream)
{
    const cudaKernel_t k = static_cast<cudaKernel_t>(h->mix_kern[(sizeof(R) == 8 ? 0 : 2) + (velocity ? 1 : 0)]);
    const cplx<R> *rt = velocity ? t.hinv : t.r;
    long long nn = (long long)t.n * t.n;
    int n = t.n, nd = t.nd, nc = t.nc;
    const cplx<R> *dcoef = t.dcoef;
    const R *ldiff = t.ldiff;
    void *args[] = {(void *)&psi, (void *)&out, (void *)&t.rad, (void *)&rt, (void *)&w1, (void *)&w2,
                    (void *)&dcoef, (void *)&ldiff, &nn, &n, &nd, &nc, (void *)&fb, &beta, &gamma};
    const unsigned point_blocks = (unsigned)std::min<long long>((nn + 127) / 128, 65535);
    const size_t smem = 2 * (size_t)std::max(nd, 1) * sizeof(cplx<R>);
    const bool one_thread_per_point = (long long)point_blocks * fb.count >= 8LL * sm_count(h->device);
    const dim3 grid(one_thread_per_point ? 1u : (unsigned)h->plan.mix.size(), point_blocks, (unsigned)fb.count);
    HE_CUDA_TRY(cudaLaunchKernel(reinterpret_cast<const void *>(k), grid, dim3(128), args, smem, stream));
    return HE_OK;
}

template int launch_mix_jit<double>(he_operator *, const DeviceTables<double> &, const double2 *, double2 *,
                                    const double2 *, const double2 *, const FieldBatch &, int, double2, double2,
                                    cudaStream_t);
template int launch_mix_jit<float>(he_operator *, const DeviceTables<float> &, const float2 *, float2 *,
                                   const float2 *, const float2 *, const FieldBatch &, int, float2, float2,
                                   cudaStream_t);

}  // namespace he

// Source of the generated mixing kernel for a plan built by he_plan_build (host only).
extern "C" long long he_plan_mix_source(void *plan, int dipole_real, char *buf, long long cap)
{
    const std::string s = he::mix_source(*static_cast<he_plan_host *>(plan), dipole_real != 0, -1);
    if (buf && cap > 0) {
        const size_t n = std::min<size_t>((size_t)cap - 1, s.size());
        memcpy(buf, s.data(), n);
        buf[n] = '\0';
    }
    return (long long)s.size();
}

// Compile a source with NVRTC for sm_100a (host only, no device needed).  Returns 0 when
// it compiles; the compiler log goes to `log`.
extern "C" int he_nvrtc_check(const char *src, char *log, long long cap)
{
    std::string l;
    const bool ok = !he::nvrtc_compile(src, l).empty();
    if (log && cap > 0) {
        const size_t n = std::min<size_t>((size_t)cap - 1, l.size());
        memcpy(log, l.data(), n);
        log[n] = '\0';
    }
    return ok ? 0 : 1;
}

// The mixing program of a planner handle as JSON (host only): groups with their output
// channels, blocks (sources, multipole terms with edges) and dipole edges per electron.
extern "C" long long he_plan_mix_program(void *plan, char *buf, long long cap)
{
    const he_plan_host &P = *static_cast<he_plan_host *>(plan);
    std::ostringstream o;
    o.precision(17);
    auto ints = [&](const std::vector<int> &v) {
        o << '[';
        for (size_t k = 0; k < v.size(); ++k) o << (k ? "," : "") << v[k];
        o << ']';
    };
    o << '[';
    for (size_t g = 0; g < P.mix.size(); ++g) {
        const MixGroup &G = P.mix[g];
        o << (g ? "," : "") << "{\"out\":";
        ints(G.out);
        o << ",\"blocks\":[";
        for (size_t b = 0; b < G.blocks.size(); ++b) {
            const MixBlock &B = G.blocks[b];
            o << (b ? "," : "") << "{\"src\":";
            ints(B.src);
            o << ",\"terms\":[";
            for (size_t t = 0; t < B.terms.size(); ++t) {
                const MixTerm &T = B.terms[t];
                o << (t ? "," : "") << "{\"lam\":" << T.lam << ",\"d\":";
                ints(T.d);
                o << ",\"s\":";
                ints(T.s);
                o << ",\"w\":[";
                for (size_t k = 0; k < T.w.size(); ++k) o << (k ? "," : "") << T.w[k];
                o << "]}";
            }
            o << "]}";
        }
        o << "],\"dip\":[";
        for (int e = 0; e < 2; ++e) {
            o << (e ? "," : "") << "{\"d\":";
            ints(G.dd[e]);
            o << ",\"s\":";
            ints(G.ds[e]);
            o << ",\"k\":";
            ints(G.dk[e]);
            o << '}';
        }
        o << "]}";
    }
    o << ']';
    const std::string s = o.str();
    if (buf && cap > 0) {
        const size_t n = std::min<size_t>((size_t)cap - 1, s.size());
        memcpy(buf, s.data(), n);
        buf[n] = '\0';
    }
    return (long long)s.size();
}
