// umma.cuh -- 5th-generation tensor-core (tcgen05) building blocks for sm_100a: tensor-memory
// allocation, shared-memory matrix descriptors, the BF16 MMA with FP32 accumulation in tensor memory,
// the commit to an mbarrier, and tensor-memory loads (PTX ISA 8.6, tcgen05.*).
//
// Operand layout in shared memory (no swizzle): a matrix T with R rows and C columns of bf16 is stored
// as core matrices of 8 rows x 8 columns (8 x 16 bytes, rows 16 bytes apart), column block first:
//
//     byte offset of T(r, c) = ((c / 8) * R + r) * 16 + (c % 8) * 2
//
// The same buffer serves as a K-major operand (rows = M or N, columns = K) or, read transposed, as an
// MN-major operand (columns = M or N, rows = K); desc_kmajor / desc_mnmajor give the two descriptors.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

#include "common.cuh"

namespace gsph {
namespace umma {

// byte offset of element (r, c) in the core-matrix layout of a matrix with R rows
__host__ __device__ __forceinline__ uint32_t off(int r, int c, int R) {
    return static_cast<uint32_t>(((c >> 3) * R + r) * 16 + (c & 7) * 2);
}

// shared-memory matrix descriptor (no swizzle): start address, leading-dimension byte offset (LBO),
// stride-dimension byte offset (SBO), descriptor version 1 (sm_100)
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// K-major operand from a buffer with R rows (rows = M/N, columns = K), k-step s of 16 columns:
// 8-row groups are 128 bytes apart (SBO), 8-column groups R * 16 bytes apart (LBO)
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t base, int R, int s) {
    return make_desc(base + static_cast<uint32_t>(2 * s * R * 16), static_cast<uint32_t>(R * 16), 128u);
}
// MN-major operand from a buffer with R rows read transposed (columns = M/N, rows = K), k-step s of
// 16 rows: 8-element M/N groups are R * 16 bytes apart (SBO), 8-row K groups 128 bytes apart (LBO)
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t base, int R, int s) {
    return make_desc(base + static_cast<uint32_t>(s * 16 * 16), 128u, static_cast<uint32_t>(R * 16));
}

// instruction descriptor of kind::f16: BF16 A and B, FP32 D, M x N, each operand K-major (0) or
// MN-major (1)
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(a_mn) << 15) |
           (static_cast<uint32_t>(b_mn) << 16) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc ? 1u : 0u)
        : "memory");
}
// arrive on `bar` when every MMA issued so far by this thread has completed
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory become visible to the tensor cores (async proxy)
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// tensor-memory allocation by one whole warp; the address lands in *slot (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this thread's tensor-memory lane (see lane_addr)
__device__ __forceinline__ void ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}
// lane of this thread in a 128-lane accumulator: warp w of each warpgroup owns lanes 32 (w % 4) .. + 31
__device__ __forceinline__ uint32_t lane_addr(uint32_t tbase, int col) {
    return tbase + (static_cast<uint32_t>(((threadIdx.x >> 5) & 3) * 32) << 16) + static_cast<uint32_t>(col);
}

// store 8 consecutive bf16 columns c0..c0+7 (c0 % 8 == 0) of row r: one 16-byte write
__device__ __forceinline__ void st8(unsigned char* buf, int r, int c0, int R, const float* v) {
    __align__(16) __nv_bfloat162 h[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
    *reinterpret_cast<uint4*>(buf + off(r, c0, R)) = *reinterpret_cast<const uint4*>(h);
}

// bounded wait on the MMA-completion barrier (phase `parity`); false, status set, when it gave up
__device__ __forceinline__ bool wait_mma(uint64_t* bar, uint32_t parity, int* status) {
    return mbar_wait_bounded(bar, parity, status);
}

}  // namespace umma
}  // namespace gsph
