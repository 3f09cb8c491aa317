// Per-operator launchers (op_kernels.cu).  Internal to the library.
#pragma once

#include <cuda_runtime.h>

namespace nuc3d {

struct RK5 {
    const double *rhs[5];
    const double *un[5];
    double *ui[5];
};

cudaError_t op_reconstruct(int scheme, int upwind, unsigned quirks, int nx, long long lines,
                           const double *in, const double *hl, const double *hr, double *out,
                           cudaStream_t st);
// CRWENO5 line solve with caller-provided scratch (2 * nx * lines doubles).
cudaError_t op_crweno_into(int upwind, int nx, long long lines, const double *in,
                           const double *hl, const double *hr, double *out, double *scratch,
                           cudaStream_t st);
// Records an error for nuc3d_last_error() and returns code (capi.cu).
int set_last_error(int code, const char *msg);
cudaError_t op_cd6(int nx, long long lines, double dx, const double *in, const double *hl,
                   const double *hr, double *out, cudaStream_t st);
// scheme: VIS_CD6 / VIS_CD2 / VIS_CD8; halos (tile, lines)
cudaError_t op_differential(int scheme, int tile, int nx, long long lines, double dx,
                            const double *in, const double *hl, const double *hr, double *out,
                            cudaStream_t st);
cudaError_t op_rk3(int stage, long long n, double dt, RK5 rk, cudaStream_t st);

}  // namespace nuc3d
