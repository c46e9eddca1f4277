// Launch entry points of the mixed-precision kernels (fenice_b200/csrc/mixed.cu, a translation unit of its own: it is
// compiled with fast single-precision math, the FP64 kernels are not).
#pragma once

#include <cuda_runtime.h>

namespace fvg {
struct StageArgs;
struct ViscArgs;

struct MixedStage {
    cudaError_t (*prepare)() = nullptr;
    cudaError_t (*launch)(const StageArgs&, int, cudaStream_t) = nullptr;
};
// the mixed stage kernel for a 2-D or 3-D mesh, a reconstruction (MUSCL, WENO3-Z, WENO5-Z) and a Riemann solver; the
// tiles are the FP64 stage kernel's (3-D: 8x8x8 cells, here 384 threads; 2-D: 16x15 cells, 256 threads)
MixedStage mixed_stage(int dim, int recon, int riemann, bool full);
// the mixed WENO5-Z stage kernel with the learned troubled-cell sensor choosing linear or WENO5-Z reconstructions
// (StageArgs::sens_flags)
MixedStage mixed_stage_gated(int dim, int riemann, bool full);
cudaError_t mixed_viscous_prepare();
cudaError_t mixed_viscous_launch(const ViscArgs& a, int nblocks, cudaStream_t s);
}   // namespace fvg
