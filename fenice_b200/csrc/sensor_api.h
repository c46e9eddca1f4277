// The sensor's refresh of a run's gate (sensor.cu): the network's flags for every (cell, axis) of the state, reduced to
// the stage kernel's tiles.
#pragma once

#include "grid.cuh"

#include <cuda_runtime.h>

namespace fvg {
// The network evaluated on every (cell, axis) of the state (flags0: 1 where the cell's reconstructions along the axis
// stay WENO5-Z, logit >= theta), then, with the troubled set grown by `radius` cells along every axis (wrapping across
// periodic axes), reduced to the stage kernel's tiles: tile_flags[a * ntiles + b] = 0 where tile b's reconstructions
// along axis a may all be linear. rows: scratch of dim x nz x ny x tiles[0] bytes. With a control block the kernels run only on the steps
// where ctl->active and ctl->steps % every == 0 (the tile flags of the last refresh stay otherwise). counts (device, may
// be null) += [linear, all] tile-axes of each refresh. A part of a decomposed mesh passes the split axis and whether its
// low / high side along it is an interface (split < 0: a whole mesh): every tile whose box reaches an interface stays
// WENO5-Z along every axis, so the tiles on both sides of an interface face reconstruct it alike.
cudaError_t sensor_refresh(const Mesh& m, const Bc& bc, const Eos<double>& eos, int dim, const double* U, const void* weights, float theta, int radius,
                           const int periodic[3], unsigned char* flags0, unsigned char* rows, const int tile[3], const int tiles[3],
                           unsigned char* tile_flags, const Ctl* ctl, int every, unsigned long long* counts, cudaStream_t s, int split = -1,
                           int peer_lo = 0, int peer_hi = 0);
}   // namespace fvg
