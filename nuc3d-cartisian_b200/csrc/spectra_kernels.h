// Shell-binned spectra of one box (spectra_kernels.cu).  Internal.
#pragma once

#include <cuda_runtime.h>

#include "rhs_kernels.h"

namespace nuc3d {

constexpr int kSpectra = 9;         // kin, kinc, kins, kinl, kinr, hel, ens, den, pre
constexpr int kSpectraFields = 7;   // transformed fields: u, v, w, hel, ens, rho, p
constexpr int kSpecBlocks = 592;    // fixed binning grid (4 x 148): results do not depend on the batch

inline int spectra_kmax(const BoxParams &p) {
    int m = p.n[0] < p.n[1] ? p.n[0] : p.n[1];
    return (m < p.n[2] ? m : p.n[2]) / 2;
}
// device scratch of a spectra evaluation: the seven complex fields, the
// per-block shell partials and the result
size_t spectra_scratch_bytes(const BoxParams &p);
// Spectra of box b (W must hold the primitives of U[0]) into
// d_out[kSpectra * kmax]; scratch of spectra_scratch_bytes.  Plans, runs and
// releases its cuFFT plan on st.  Returns a CUDA error, or
// cudaErrorUnknown with *fft_status set when cuFFT fails.
cudaError_t launch_spectra(const BoxDev &b, void *scratch, double *d_out, int *fft_status,
                           cudaStream_t st);

}  // namespace nuc3d
