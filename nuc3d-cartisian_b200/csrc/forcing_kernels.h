// Spectral shell forcing (forcing_kernels.cu).  Internal.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "rhs_kernels.h"

namespace nuc3d {

// PhysModel.in Forcing_amplitude, Forcing_amplitude_hel, Forcing_wave_k
// (physicsModel.cpp:1422-1424); K = floor(k + 1/2) bounds |k_d| of the shell.
// band = 1: the band forcing at a fixed injection rate (NUC3D_FORCING_BAND):
// amp is the injection rate P and k the band radius.
struct ForceParams {
    double amp, hel, k;
    int K;
    int band;
};

// Device scratch of one forced box (one allocation, laid out by forcing_layout).
struct ForceScratch {
    double2 *tx, *ty, *tz;  // twiddles exp(+i 2 pi k j / n), k = -K..K
    double2 *a, *b, *fh;    // transform passes and the forcing spectrum
    double *partials;       // per-line sums of f.u
    double *scal;           // E_s, E_c, theta (band: the gain P / (2 E_b)), <f.u>
};

constexpr int kForceMaxK = 3;  // shells up to k_f < 3.5
int forcing_K(double k_f);
size_t forcing_scratch_bytes(const BoxParams &p, double k_f);
ForceScratch forcing_layout(const BoxParams &p, double k_f, void *base);
// twiddle tables (once per box)
cudaError_t forcing_prepare(const BoxParams &p, double k_f, const ForceScratch &s, cudaStream_t st);
// R[1..4] of the box -= the forcing of its current primitives W (Bk: bulk type of R)
template <typename Bk>
cudaError_t launch_forcing(const BoxDev &b, const ForceScratch &s, ForceParams fp, cudaStream_t st);

}  // namespace nuc3d
