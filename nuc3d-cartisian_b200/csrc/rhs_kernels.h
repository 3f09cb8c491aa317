// Host-side launch interface of the whole-box kernels (rhs_kernels.cu,
// crweno_kernels.cu).  Internal to the library; the public surface is the C
// ABI in include/nuc3d_b200.h.
#pragma once

#include <cuda_runtime.h>

#include "nuc3d_device.cuh"

namespace nuc3d {

constexpr int kHistory = 1024;  // per-call step history kept on the device

struct StateView {
    const double *q[5];
};
struct StateViewMut {
    double *q[5];
};
struct PrimView {
    double *w[6];  // u, v, w, p, c, T  (FP64)
};
template <typename B>
struct BView {
    B *f[5];
};
template <typename B>
struct BView9 {
    B *f[9];
};

// Per-box scalars that live in device memory so a step never waits on the
// host: dt of the current step, accumulated time, and per-step history.
struct StepScalars {
    double dt;
    double dt_local;
    double time;
    double pad;
    double dt_hist[kHistory];
    double res_hist[kHistory];
};

cudaError_t launch_prim(const BoxParams &bp, StateView q, PrimView w, double *eig, int want_eig,
                        int sms, cudaStream_t st);
cudaError_t launch_dt(const BoxParams &bp, const double *eig, StepScalars *sc, int step,
                      cudaStream_t st);
template <typename B>
cudaError_t launch_inviscid(const BoxParams &bp, int dir, StateView q, PrimView w, BView<B> r,
                            int accumulate, cudaStream_t st);
template <typename B>
cudaError_t launch_visc_flux(const BoxParams &bp, PrimView w, BView9<B> vf, int sms,
                             cudaStream_t st);
// stage 0..2: TVD-RK3 update into uout; stage -1: uout receives the total RHS.
template <typename B>
cudaError_t launch_update(const BoxParams &bp, BView<B> r, BView9<B> vf, StateView un,
                          StateView uin, StateViewMut uout, int stage, const StepScalars *sc,
                          double *res_acc, unsigned *flags, int sms, cudaStream_t st);
cudaError_t launch_residual(const BoxParams &bp, StepScalars *sc, double *res_acc, int step,
                            cudaStream_t st);

// CRWENO5 whole-box sweep (crweno_kernels.cu).  scratch: 2 * lines * n bulk
// values for the forward-sweep coefficients.
template <typename B>
cudaError_t launch_crweno(const BoxParams &bp, int dir, StateView q, PrimView w, BView<B> r,
                          int accumulate, B *scratch, cudaStream_t st, int *nlaunch);
size_t crweno_scratch_elems(const BoxParams &bp);

}  // namespace nuc3d
