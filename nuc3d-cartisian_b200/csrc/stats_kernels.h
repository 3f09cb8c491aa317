// Device turbulence statistics of one box (stats_kernels.cu).  Internal.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "rhs_kernels.h"

namespace nuc3d {

constexpr int kStatsSums = 23;     // per-cell sums accumulated on the device
constexpr int kStatsBlocks = 296;  // fixed grid: the sums do not depend on the batch
constexpr int kStatsOut = 26;      // values reported (NUC3D_STATS)

// Scratch of (1 + kStatsBlocks) * kStatsSums doubles; W must hold the
// primitives of U[0].  The kStatsSums totals land at scratch[0..].
cudaError_t launch_stats(const BoxDev &b, double *scratch, cudaStream_t st);
// The reported values from the totals (postproc.cpp:855-876).
void stats_finish(const BoxParams &p, const double *sums, double *out);
constexpr size_t stats_scratch_doubles() { return (size_t)(1 + kStatsBlocks) * kStatsSums; }

}  // namespace nuc3d
