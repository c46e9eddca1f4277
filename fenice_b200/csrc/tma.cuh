// Tensor-memory-accelerator (TMA) staging of a stage tile's box: the tensor maps of a state's planes and the PTX of the
// bulk tensor copy and of the shared-memory barrier that completes it.
//
// A state of nvar FP64 planes is a 4-D tensor (x, y, z, plane): dims (nx, ny, nz, nvar), byte strides (8 nx, 8 nx ny,
// 8 plane). The mixed stage kernel reads the 8x8x8 tile with 3 cells beyond its faces: a 16 x 8 x 8 box starting at
// x = o - 4 (the tile and its x halos; the start of a TMA box must lie on 16 bytes, an even cell index for 8-byte
// values), and either 8 x 14 x 8 / 8 x 8 x 14 boxes (the per-axis sweep) or 8 x 3 x 8 / 8 x 8 x 3 boxes (the halos of the
// cross). Only boxes inside the mesh are copied (wrapped, ghost and forced cells need the index-mapping loader), and no
// copy here ever multicasts.
#pragma once

#include <cuda.h>

namespace fvg {

// the maps of one state buffer (passed to the kernel as a __grid_constant__ parameter): the 16 x 8 x 8 box, the per-axis
// sweep's 8 x 14 x 8 and 8 x 8 x 14 boxes, the cross's 8 x 3 x 8 and 8 x 8 x 3 halo boxes
struct TmaMaps {
    CUtensorMap m[5];
};

namespace tma {
__device__ __forceinline__ unsigned su32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// the copy's bytes the barrier's phase waits for (one arrival, by the issuing thread)
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// generic-proxy accesses to shared memory before an async-proxy (TMA) write to the same bytes
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// the box at (x, y, z, plane) of a 4-D map into shared memory (128-byte aligned), completing on `bar`
__device__ __forceinline__ void load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int q, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(su32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(q), "r"(su32(bar))
        : "memory");
}
}   // namespace tma

}   // namespace fvg
