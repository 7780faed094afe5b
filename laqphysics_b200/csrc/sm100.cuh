// Blackwell (sm_100a) primitives written as inline PTX: mbarriers with bounded waits,
// 2-D TMA tile loads, tcgen05 tensor-memory allocation, the tcgen05.mma issue of the
// TF32 kind with shared-memory operand descriptors, commit to an mbarrier, and tensor
// memory loads for the epilogue.  Used by the separable preconditioner's TF32 GEMMs.
//
// Layout conventions (PTX ISA, tcgen05 "matrix descriptors"): both operands are K-major
// tiles whose rows are one 128-byte swizzle atom wide (32 fp32 values of K), written by a
// TMA load with CU_TENSOR_MAP_SWIZZLE_128B; 8 consecutive rows form a 1024-byte group
// (the stride byte offset), and a K slice of 8 values (one MMA) starts 32 bytes further
// into the atom.  Every tile base is 1024-byte aligned so the swizzle phase is zero.
#pragma once
#include <cuda.h>
#include <stdint.h>

namespace he {
namespace sm100 {

constexpr int WAIT_LIMIT = 1 << 22;              // try_wait rounds before a wait counts as lost
constexpr unsigned WAIT_HINT_NS = 1000;          // suspend hint of one try_wait round

__device__ __forceinline__ unsigned saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void bar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity), "r"(WAIT_HINT_NS)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar` to complete; false when the iteration limit ran out.
__device__ __forceinline__ bool bar_wait(uint64_t *bar, unsigned parity)
{
    for (int k = 0; k < WAIT_LIMIT; ++k)
        if (bar_try_wait(bar, parity)) return true;
    return false;
}

// One 2-D tiled TMA load (box of the tensor map at element coordinates x, y), completing
// its bytes on `bar`.  x * 4 bytes must be a multiple of 16 (callers pass multiples of 32).
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(saddr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ---- tensor memory ------------------------------------------------------------------
// Allocation by one whole warp; the TMEM base address is written to *slot (shared).
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, unsigned columns)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(slot)), "r"(columns)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t base, unsigned columns)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(columns) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- operand descriptors and the MMA --------------------------------------------------
// K-major tile, 128-byte swizzle: start address, leading byte offset 16 (unused for this
// layout), stride byte offset 1024 (8 rows of 128 bytes), descriptor version 1, swizzle 2.
__device__ __forceinline__ uint64_t desc_k_sw128(unsigned smem_address)
{
    uint64_t d = (uint64_t)((smem_address >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor of kind::tf32: fp32 accumulator, TF32 A and B, both K-major,
// M = 128 rows, N columns (a multiple of 16, at most 256).
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, int accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive on `bar` once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

// 32 consecutive fp32 columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31).
__device__ __forceinline__ void tmem_load32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

// Round to the nearest TF32 value (10 explicit mantissa bits), ties away from zero.
__device__ __forceinline__ float tf32_round(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

}  // namespace sm100
}  // namespace he
