// Device generators of initial states (init_kernels.cu).  Internal.
#pragma once

#include <cuda_runtime.h>

#include "rhs_kernels.h"

namespace nuc3d {

// Retained wavenumbers of one axis of the HIT synthesis: k = kmin .. kmin+M-1
// (|k| <= 6.5 kp, and the FFT index set of n points), kscale = 2 pi / L.
struct HitAxis {
    int n, M, kmin, pad;
    double kscale;
};
HitAxis hit_axis(int n, double length, double k_peak);
// Device scratch the HIT synthesis of a box needs.
size_t hit_scratch_bytes(const BoxParams &p, double k_peak);

// U[0] of the box <- Taylor-Green vortex on the cell centres.
cudaError_t launch_init_tgv(const BoxDev &b, cudaStream_t st);
// Raw random-phase velocity into W[0..2] of the box and six sums into d_sums:
// sum u^2, v^2, w^2, (du/dx)^2, (dv/dy)^2, (dw/dz)^2 over the cells.
cudaError_t launch_hit_synthesis(const BoxDev &b, double lx, double ly, double lz,
                                 unsigned long long seed, double k_peak, double u_rms,
                                 void *scratch, double *d_sums, cudaStream_t st);
// U[0] <- rho = 1, velocity = scale * W[0..2], p = 1 / (gamma M^2).
cudaError_t launch_hit_finalize(const BoxDev &b, double scale, cudaStream_t st);

}  // namespace nuc3d
