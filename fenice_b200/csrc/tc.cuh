// The fifth-generation tensor cores (tcgen05) for the learned sensor's dense layers: bf16 operands in shared memory,
// f32 accumulators in tensor memory (TMEM), one thread issuing the MMA and a shared-memory barrier signalled by
// tcgen05.commit when it completes.
//
// Operand layout (the "no swizzle" canonical K-major layout of the MMA's shared-memory matrix descriptor): an R x 32
// bf16 matrix (R rows, K = 32) is stored as core matrices of 8 rows x 8 elements (16 bytes per row, 128 bytes each),
// core matrix (row / 8, k / 8) at byte (row / 8 * 4 + k / 8) * 128. One MMA takes K = 16: the two core matrices along K
// are 128 bytes apart (the descriptor's leading byte offset), consecutive 8-row groups 512 bytes apart (its stride byte
// offset), and the k-step s starts 256 s bytes in. The descriptor and instruction-descriptor bit fields follow the
// PTX ISA's tcgen05 matrix and instruction descriptors (the same fields CUTLASS's cute/arch/mma_sm100_desc.hpp names).
#pragma once

#include <stdint.h>

namespace fvg {
namespace tc {

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// element offset of (row, k) of an R x 32 bf16 matrix in the canonical layout
__device__ __forceinline__ int cl_index(int row, int k) { return ((row >> 3) * 4 + (k >> 3)) * 64 + (row & 7) * 8 + (k & 7); }

// shared-memory matrix descriptor of k-step s (K = 16) of a canonical R x 32 bf16 matrix at `base` (16-byte aligned):
// start address, leading byte offset 128, stride byte offset 512 (all in 16-byte units), descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(const void* base, int s) {
    const uint64_t addr = (uint64_t)((su32(base) + 256u * (uint32_t)s) >> 4) & 0x3FFFull;
    return addr | (uint64_t(128 >> 4) << 16) | (uint64_t(512 >> 4) << 32) | (1ull << 46);
}

// a matrix descriptor with explicit byte offsets: start `base` + `off`, leading byte offset `lbo` (between the core
// matrices adjacent along K for a K-major operand, along K too for an MN-major one), stride byte offset `sbo` (between
// the core matrices adjacent along M or N); no swizzle
__device__ __forceinline__ uint64_t smem_desc_at(const void* base, uint32_t off, uint32_t lbo, uint32_t sbo) {
    const uint64_t addr = (uint64_t)((su32(base) + off) >> 4) & 0x3FFFull;
    return addr | (uint64_t((lbo >> 4) & 0x3FFF) << 16) | (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: f32 accumulator, bf16 A and B, N columns, M rows; A and B K-major (MN_MAJOR
// false) or both MN-major
template <int M, int N, bool MN_MAJOR = false> __host__ __device__ constexpr uint32_t idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (MN_MAJOR ? (1u << 15) | (1u << 16) : 0u) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// TMEM allocation of `cols` columns (a power of two >= 32) by one whole warp; the address lands in *slot (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(slot)), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// D (TMEM) = A B^T (+ D when accumulate): A M x 16, B N x 16 from shared-memory descriptors; issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate ? 1u : 0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// the shared-memory barrier `bar` receives one arrival when every tcgen05 operation this thread issued has completed
__device__ __forceinline__ void commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar)) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// the 32 f32 columns col .. col + 31 of TMEM lane (32 * (warp % 4) + lane) into v (a whole warp; the warp reads its own
// quarter of the lanes); the wait for the load is in the same asm statement, so no use of v precedes it
__device__ __forceinline__ void ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, "
        "%20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]),
          "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

}   // namespace tc
}   // namespace fvg
