// The mixed-precision kernels' translation unit (see mixed.cuh). Built with --use_fast_math: FP32 division and square
// root are the fast approximations and multiplies and adds may contract into FMAs, except where mixed.cuh rounds each
// operation explicitly (the face values, the balance, the FP64 update); FP64 division and square root stay IEEE.
#include "mixed.cuh"
#include "mixed_api.h"

namespace fvg {
namespace {

template <int DIM> struct MTile;
// 3-D: 384 threads per 8x8x8 tile, three CTAs per SM (36 warps; 2.85 ms per launch at 256^3 against 3.52 with 192 threads)
template <> struct MTile<3> { static constexpr int X = 8, Y = 8, Z = 8, NT = 384; };
template <> struct MTile<2> { static constexpr int X = 16, Y = 15, Z = 1, NT = 256; };

// the cross-box kernel whose tiles inside the mesh come in by TMA: the 3-D WENO5-Z lean kernels, when the run passes
// tensor maps (StageArgs::tma); 8x8x8 tiles of 384 threads
template <int DIM, int RECON, bool FULL> constexpr bool kHasTma = DIM == 3 && RECON == kWeno5 && !FULL;

template <int RIEMANN, bool GATED> struct TmaK {
    static constexpr int NT = MTile<3>::NT;
    static_assert(MTile<3>::X == 8 && MTile<3>::Y == 8 && MTile<3>::Z == 8, "the cross-box kernel's tile");
    static cudaError_t prepare() {
        return cudaFuncSetAttribute(mixed_stage_kernel_tma<RIEMANN, NT, GATED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CrossShape::SMEM_BYTES);
    }
    static cudaError_t launch(const StageArgs& a, int nblocks, cudaStream_t s) {
        mixed_stage_kernel_tma<RIEMANN, NT, GATED><<<nblocks, NT, CrossShape::SMEM_BYTES, s>>>(a, *static_cast<const TmaMaps*>(a.tma));
        return cudaGetLastError();
    }
};

template <int DIM, int RECON, int RIEMANN, bool FULL> struct MixedK {
    using T = MTile<DIM>;
    using S = MixedShape<DIM, RECON, T::X, T::Y, T::Z>;
    static cudaError_t prepare() {
        cudaError_t e = cudaFuncSetAttribute(mixed_stage_kernel<DIM, RECON, RIEMANN, T::X, T::Y, T::Z, T::NT, false, FULL>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM_BYTES);
        if constexpr (kHasTma<DIM, RECON, FULL>)
            if (e == cudaSuccess) e = TmaK<RIEMANN, false>::prepare();
        return e;
    }
    static cudaError_t launch(const StageArgs& a, int nblocks, cudaStream_t s) {
        if constexpr (kHasTma<DIM, RECON, FULL>)
            if (a.tma) return TmaK<RIEMANN, false>::launch(a, nblocks, s);
        mixed_stage_kernel<DIM, RECON, RIEMANN, T::X, T::Y, T::Z, T::NT, false, FULL><<<nblocks, T::NT, S::SMEM_BYTES, s>>>(a);
        return cudaGetLastError();
    }
};

// the WENO5-Z kernels gated by the learned sensor
template <int DIM, int RIEMANN, bool FULL> struct GatedK {
    using T = MTile<DIM>;
    using S = MixedShape<DIM, kWeno5, T::X, T::Y, T::Z>;
    static cudaError_t prepare() {
        cudaError_t e = cudaFuncSetAttribute(mixed_stage_kernel<DIM, kWeno5, RIEMANN, T::X, T::Y, T::Z, T::NT, true, FULL>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM_BYTES);
        if constexpr (kHasTma<DIM, kWeno5, FULL>)
            if (e == cudaSuccess) e = TmaK<RIEMANN, true>::prepare();
        return e;
    }
    static cudaError_t launch(const StageArgs& a, int nblocks, cudaStream_t s) {
        if constexpr (kHasTma<DIM, kWeno5, FULL>)
            if (a.tma) return TmaK<RIEMANN, true>::launch(a, nblocks, s);
        mixed_stage_kernel<DIM, kWeno5, RIEMANN, T::X, T::Y, T::Z, T::NT, true, FULL><<<nblocks, T::NT, S::SMEM_BYTES, s>>>(a);
        return cudaGetLastError();
    }
};

template <int DIM, int RECON, bool FULL> MixedStage pick_r(int riemann) {
    if (riemann == kLowMach) return {MixedK<DIM, RECON, kLowMach, FULL>::prepare, MixedK<DIM, RECON, kLowMach, FULL>::launch};
    return {MixedK<DIM, RECON, kHLLC, FULL>::prepare, MixedK<DIM, RECON, kHLLC, FULL>::launch};
}
template <int DIM, bool FULL> MixedStage pick(int recon, int riemann) {
    switch (recon) {
    case kMuscl: return pick_r<DIM, kMuscl, FULL>(riemann);
    case kWeno3: return pick_r<DIM, kWeno3, FULL>(riemann);
    default: return pick_r<DIM, kWeno5, FULL>(riemann);
    }
}
template <int DIM, bool FULL> MixedStage pick_gated(int riemann) {
    return riemann == kLowMach ? MixedStage{GatedK<DIM, kLowMach, FULL>::prepare, GatedK<DIM, kLowMach, FULL>::launch}
                               : MixedStage{GatedK<DIM, kHLLC, FULL>::prepare, GatedK<DIM, kHLLC, FULL>::launch};
}

}   // namespace

// full: the kernels with the code of part interfaces and non-reflecting sides; else the lean instantiation
MixedStage mixed_stage(int dim, int recon, int riemann, bool full) {
    if (dim == 3) return full ? pick<3, true>(recon, riemann) : pick<3, false>(recon, riemann);
    return full ? pick<2, true>(recon, riemann) : pick<2, false>(recon, riemann);
}

MixedStage mixed_stage_gated(int dim, int riemann, bool full) {
    if (dim == 3) return full ? pick_gated<3, true>(riemann) : pick_gated<3, false>(riemann);
    return full ? pick_gated<2, true>(riemann) : pick_gated<2, false>(riemann);
}

// the FP32 viscous sweep: 384 threads per 8x8x8 tile (1.15 ms per launch at 256^3 against 1.28 with 192 threads); the
// instantiation without the ghost rules and wall tests when every side of the launch is periodic or a part interface
constexpr int kMixedViscNT = 384;
cudaError_t mixed_viscous_prepare() {
    cudaError_t e = cudaFuncSetAttribute(mixed_viscous_kernel<8, 8, 8, kMixedViscNT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)MixedViscShape<8, 8, 8>::SMEM_BYTES);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(mixed_viscous_kernel<8, 8, 8, kMixedViscNT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)MixedViscShape<8, 8, 8>::SMEM_BYTES);
    return e;
}
cudaError_t mixed_viscous_launch(const ViscArgs& a, int nblocks, cudaStream_t s) {
    bool walls = false;
    for (int side = 0; side < 6; ++side) walls = walls || !a.through[side];
    if (walls)
        mixed_viscous_kernel<8, 8, 8, kMixedViscNT, true><<<nblocks, kMixedViscNT, MixedViscShape<8, 8, 8>::SMEM_BYTES, s>>>(a);
    else
        mixed_viscous_kernel<8, 8, 8, kMixedViscNT, false><<<nblocks, kMixedViscNT, MixedViscShape<8, 8, 8>::SMEM_BYTES, s>>>(a);
    return cudaGetLastError();
}

}   // namespace fvg
