// Minimal sm_100a tensor-core (tcgen05) primitives used by the split-BF16 readout: tensor-memory allocation,
// the shared-memory matrix descriptor, the kind::f16 instruction descriptor, MMA issue, commit to an mbarrier,
// and the tensor-memory load. Descriptor bit layouts follow the PTX ISA (and CUTLASS's cute/arch/
// mma_sm100_desc.hpp, which spells out the same fields).
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "bloch_common.cuh"

// Shared-memory matrix descriptor, no swizzle, K-major ("interleaved") canonical layout: core matrices of 8 rows
// x 16 bytes (8 bf16 along K, rows 16 bytes apart); `lbo` = byte distance between the two K-adjacent core
// matrices of one K=16 step, `sbo` = byte distance between 8-row groups. Bits: start >> 4 [0,14), lbo >> 4
// [16,30), sbo >> 4 [32,46), version 1 [46,48), base offset 0, layout type 0 (no swizzle) [61,64).
__device__ __forceinline__ uint64_t umma_desc(uint32_t smem_addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of tcgen05.mma kind::f16: D float32, A and B bfloat16 (both: mixing f16 and bf16
// operands is not allowed), both K-major, shape M x N (M in {64, 128}, N a multiple of 16 for M = 128).
__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int m, int n) {
    return (1u << 4)                      // D format: F32
           | (1u << 7)                    // A format: BF16
           | (1u << 10)                   // B format: BF16
           | ((uint32_t)(n >> 3) << 17)   // N >> 3
           | ((uint32_t)(m >> 4) << 24);  // M >> 4
}

// D[tmem] (+)= A[smem] . B[smem]^T, issued by one thread; `accumulate` 0 overwrites D.
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive on `bar` once every tcgen05.mma issued so far by this thread has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Tensor-memory allocation of `ncols` columns (a power of two >= 32) by one full warp; the base address is
// written to shared memory at `dst`.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit columns of this thread's tensor-memory lane (warp w reads lanes 32 w .. 32 w + 31;
// the lane offset is in bits [16, 32) of the address). Complete with tmem_ld_wait().
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// float -> (hi, lo) bfloat16 pair: hi = bf16(x) (round to nearest), lo = bf16(x - hi); hi + lo carries 16 bits.
__device__ __forceinline__ void split_bf16(float x, uint16_t& hi, uint16_t& lo) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}
