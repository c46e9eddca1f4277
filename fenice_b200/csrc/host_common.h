// Host-side helpers of the single runs (runtime.cu) that the batched runs (batch.cu) share.
#pragma once

#include "../../include/fenice_gpu.h"
#include "grid.cuh"

#include <cuda_runtime.h>
#include <string>

namespace fvg {
// why a configuration cannot run on the device ("" when it can)
std::string config_error(const fvg_config& c);
// whether it has case-file source terms or time-dependent boundary values
bool config_has_expressions(const fvg_config& c);
// the halo kind (kHalo*) of each side for a reconstruction `depth` cells deep
void config_halo_kinds(const fvg_config& c, int depth, int kinds[6]);
// the message fvg_create_error() returns (this thread's)
std::string* create_error_slot();

// What the sensor's data extraction reads of a single run: its mesh, boundary conditions, gas, current state planes,
// stream and WENO epsilon.
struct RunView {
    Mesh m;
    Bc bc;
    Eos<double> eos;
    const double* U;
    cudaStream_t stream;
    int dim, nvar, device;
    double weno_eps;
};
bool run_view(fvg_run* run, RunView* v);
}   // namespace fvg
