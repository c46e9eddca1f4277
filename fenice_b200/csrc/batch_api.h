// Launch entry points of the batched stage kernels: the FP64 ones (batch.cu, IEEE-rounded FP64) and the mixed-precision
// ones (batch_mixed.cu, compiled with fast single-precision math), each for one tile shape of kBatchShape, a
// reconstruction and a Riemann solver.
#pragma once

#include <cuda_runtime.h>

namespace fvg {
struct BatchArgs;

struct BatchStage {
    cudaError_t (*prepare)() = nullptr;                                  // raise the kernel's shared-memory limit
    cudaError_t (*launch)(const BatchArgs&, int grid, cudaStream_t) = nullptr;
    int (*resident)() = nullptr;                                         // CTAs of the kernel one SM holds
};
BatchStage batch_fp64_stage(int shape, int recon, int riemann);
BatchStage batch_mixed_stage(int shape, int recon, int riemann);
}   // namespace fvg
