// Blackwell (sm_100a) tensor-core plumbing shared by the tensor-core kernels
// of librcabf: mbarriers with bounded waits, 2-D TMA tile loads, tcgen05.mma
// (kind::f16, A operand in tensor memory, B operand in shared memory),
// tcgen05.commit, tensor-memory stores / loads, and the shared-memory and
// instruction descriptors (PTX ISA, "tcgen05" and "cp.async.bulk.tensor").
//
// Descriptor formats (64-bit shared-memory matrix descriptor of tcgen05):
//   bits  0-13  start address >> 4
//   bits 16-29  leading-dimension byte offset >> 4
//   bits 32-45  stride-dimension byte offset >> 4
//   bits 46-47  version (1 on sm_100)
//   bits 49-51  base offset (0: swizzle atoms 1024-byte aligned)
//   bit  52     leading-offset mode (0)
//   bits 61-63  layout: 0 none, 2 128-byte swizzle, 4 64-byte, 6 32-byte
// For an MN-major operand with the 128-byte swizzle, a swizzle atom is 8 rows
// (K) of 128 bytes (64 16-bit elements along MN), rows 128 bytes apart; the
// leading offset is the step between atoms along MN, the stride offset the
// step between groups of 8 rows along K.
// Instruction descriptor of kind::f16 (32-bit):
//   bits 4-5 accumulator format (1: F32), bits 7-9 / 10-12 A / B format
//   (0: F16, 1: BF16), bit 15 / 16 A / B major (0: K, 1: MN), bits 17-22
//   N >> 3, bits 24-28 M >> 4.
// A 16-bit A operand in tensor memory (M = 128): row m in lane m, element k
// in column k / 2 (even k in the low half of the 32-bit cell).
#pragma once

#include <cstdint>

#include "rcabf_internal.h"
#include "tmem.cuh"

namespace rcabf {

// ------------------------------------------------------------------------
// mbarrier
// ------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Whether the phase of `bar` with the given parity has completed (no wait).
__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for the phase of `bar` with the given parity to complete, for at
// most `limit_ns` nanoseconds, or until *abort is set by another thread.
// Returns false (and sets *abort) when it gives up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort,
                                          uint64_t limit_ns = 2000000000ull)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort) return false;
        if (global_ns() - t0 > limit_ns) {
            *abort = 1;
            return false;
        }
    }
}

// ------------------------------------------------------------------------
// TMA: 2-D tile load global -> shared, completion counted on an mbarrier
// ------------------------------------------------------------------------
__device__ __forceinline__ void tma_prefetch_desc(const void *tmap)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tmap)) : "memory");
}
// x: innermost coordinate (elements), y: row.  The caller keeps x * element
// size a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(void *dst, const void *tmap, uint64_t *bar, int32_t x, int32_t y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
        "[%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// 3-D tile load, coordinates (x, y, z) innermost first
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, uint64_t *bar, int32_t x, int32_t y,
                                            int32_t z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// ------------------------------------------------------------------------
// tcgen05: MMA, commit, tensor-memory stores
// ------------------------------------------------------------------------
// D[tmem] (+)= A[tmem] * B[smem desc], kind::f16, single CTA
__device__ __forceinline__ void umma_f16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                            uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}"
        ::"r"(d_tmem), "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// arrives once on `bar` when every MMA this thread issued before has completed
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
// r[0..7] -> 8 consecutive columns of this thread's lane
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr), "r"(r[0]),
        "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
        : "memory");
}

// ------------------------------------------------------------------------
// Descriptors
// ------------------------------------------------------------------------
// MN-major operand, 128-byte swizzle, atoms 1024-byte aligned
__device__ __forceinline__ uint64_t sdesc_mn_sw128(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}
// kind::f16, F16 x F16 (bf16: BF16 x BF16) -> F32, A K-major, B MN-major, M x N
constexpr RCABF_HD uint32_t idesc_f16_kmaj_a_mnmaj_b(int m, int n, bool bf16 = false)
{
    const uint32_t fmt = bf16 ? 1u : 0u;
    return (1u << 4) | (fmt << 7) | (fmt << 10) | (0u << 15) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

}  // namespace rcabf
