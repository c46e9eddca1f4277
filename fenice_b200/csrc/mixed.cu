// The mixed-precision kernels' translation unit (see mixed.cuh). Built with --use_fast_math: FP32 division and square
// root are the fast approximations and multiplies and adds contract into FMAs; FP64 arithmetic keeps IEEE rounding.
#include "mixed.cuh"
#include "mixed_api.h"

namespace fvg {
namespace {

template <int DIM> struct MTile;
template <> struct MTile<3> { static constexpr int X = 8, Y = 8, Z = 8, NT = 192; };
template <> struct MTile<2> { static constexpr int X = 16, Y = 15, Z = 1, NT = 256; };

template <int DIM, int RECON, int RIEMANN> struct MixedK {
    using T = MTile<DIM>;
    using S = MixedShape<DIM, RECON, T::X, T::Y, T::Z>;
    static cudaError_t prepare() {
        return cudaFuncSetAttribute(mixed_stage_kernel<DIM, RECON, RIEMANN, T::X, T::Y, T::Z, T::NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)S::SMEM_BYTES);
    }
    static cudaError_t launch(const StageArgs& a, int nblocks, cudaStream_t s) {
        mixed_stage_kernel<DIM, RECON, RIEMANN, T::X, T::Y, T::Z, T::NT><<<nblocks, T::NT, S::SMEM_BYTES, s>>>(a);
        return cudaGetLastError();
    }
};

// the WENO5-Z kernels gated by the learned sensor
template <int DIM, int RIEMANN> struct GatedK {
    using T = MTile<DIM>;
    using S = MixedShape<DIM, kWeno5, T::X, T::Y, T::Z>;
    static cudaError_t prepare() {
        return cudaFuncSetAttribute(mixed_stage_kernel<DIM, kWeno5, RIEMANN, T::X, T::Y, T::Z, T::NT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)S::SMEM_BYTES);
    }
    static cudaError_t launch(const StageArgs& a, int nblocks, cudaStream_t s) {
        mixed_stage_kernel<DIM, kWeno5, RIEMANN, T::X, T::Y, T::Z, T::NT, true><<<nblocks, T::NT, S::SMEM_BYTES, s>>>(a);
        return cudaGetLastError();
    }
};

template <int DIM, int RECON> MixedStage pick_r(int riemann) {
    if (riemann == kLowMach) return {MixedK<DIM, RECON, kLowMach>::prepare, MixedK<DIM, RECON, kLowMach>::launch};
    return {MixedK<DIM, RECON, kHLLC>::prepare, MixedK<DIM, RECON, kHLLC>::launch};
}
template <int DIM> MixedStage pick(int recon, int riemann) {
    switch (recon) {
    case kMuscl: return pick_r<DIM, kMuscl>(riemann);
    case kWeno3: return pick_r<DIM, kWeno3>(riemann);
    default: return pick_r<DIM, kWeno5>(riemann);
    }
}

}   // namespace

MixedStage mixed_stage(int dim, int recon, int riemann) { return dim == 3 ? pick<3>(recon, riemann) : pick<2>(recon, riemann); }

MixedStage mixed_stage_gated(int dim, int riemann) {
    if (dim == 3) return riemann == kLowMach ? MixedStage{GatedK<3, kLowMach>::prepare, GatedK<3, kLowMach>::launch}
                                             : MixedStage{GatedK<3, kHLLC>::prepare, GatedK<3, kHLLC>::launch};
    return riemann == kLowMach ? MixedStage{GatedK<2, kLowMach>::prepare, GatedK<2, kLowMach>::launch}
                               : MixedStage{GatedK<2, kHLLC>::prepare, GatedK<2, kHLLC>::launch};
}

cudaError_t mixed_viscous_prepare() {
    return cudaFuncSetAttribute(mixed_viscous_kernel<8, 8, 8, 192>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)MixedViscShape<8, 8, 8>::SMEM_BYTES);
}
cudaError_t mixed_viscous_launch(const ViscArgs& a, int nblocks, cudaStream_t s) {
    mixed_viscous_kernel<8, 8, 8, 192><<<nblocks, 192, MixedViscShape<8, 8, 8>::SMEM_BYTES, s>>>(a);
    return cudaGetLastError();
}

}   // namespace fvg
