// con2prim of one cell and the running eigenvalue maxima, shared by k_prim,
// the WENO x sweep (which recovers the primitives of its tiles while
// staging) and the CRWENO5 / hccs x-line sweep (whose blocks own whole
// x lines): every path computes bitwise the same W.
#pragma once

#include "nuc3d_device.cuh"
#include "rhs_kernels.h"

namespace nuc3d {

// physicsModel::con2prim (physicsModel.cpp:324-356) of one cell, FP64, with
// one reciprocal of rho (drcp_nr, within an ulp) in place of the reference's
// five divisions (each result within an ulp or two of the reference's).  k_prim
// and the x sweep (which recovers the primitives of its tile while staging)
// share it, so both give bitwise the same W.
struct PrimConst {
    double gamma, gm1, gM2;
    bool fabs_p;
    __device__ explicit PrimConst(const BoxParams &bp)
        : gamma(bp.gamma), gm1(bp.gamma - 1.0), gM2(bp.gamma * bp.mach * bp.mach),
          fabs_p((bp.quirks & QK_FABS_PRESSURE) != 0) {}
};
struct PrimCell {
    double u, v, w, p, c, T;
};
__device__ __forceinline__ void prim_cell(const PrimConst &k, const double Q[5], PrimCell &o) {
    const double ri = drcp_nr(Q[0]);
    o.u = mul_(Q[1], ri);
    o.v = mul_(Q[2], ri);
    o.w = mul_(Q[3], ri);
    // p = (E - rho/2 (u^2 + v^2 + w^2)) (gamma - 1)
    const double q2 = fma_(o.w, o.w, fma_(o.v, o.v, mul_(o.u, o.u)));
    double p = mul_(fma_(mul_(-0.5, Q[0]), q2, Q[4]), k.gm1);
    if (k.fabs_p) p = fabs(p);
    o.p = p;
    const double pr = mul_(p, ri);
    o.c = sqrt(mul_(k.gamma, pr));
    o.T = mul_(k.gM2, pr);
}
__device__ __forceinline__ void prim_store(const BoxDev &bd, long long g, const PrimCell &o) {
    double *const w = fieldW(bd, 0);
    const long long np = bd.np;
    w[g] = o.u;
    w[np + g] = o.v;
    w[2 * np + g] = o.w;
    w[3 * np + g] = o.p;
    w[4 * np + g] = o.c;
    w[5 * np + g] = o.T;
}
// the running maxEigen of RiemannLF (physicsModel.cpp:546-547, 600-601,
// 653-654) reduced over a block and folded into the box's maxima
__device__ __forceinline__ void eig_block_max(const BoxDev &bd, double lx, double ly, double lz) {
    const BoxParams &bp = bd.p;
    if ((bp.quirks & QK_ZETA_EIGEN) && bp.riemann == RIEMANN_LF) {
        // RiemannLF's z loop writes MaxEigen_eta; zeta stays 0 (the AUSM
        // loops keep their own directions)
        ly = fmax(lz, ly);
        lz = 0.0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        lx = fmax(lx, __shfl_xor_sync(0xffffffffu, lx, o));
        ly = fmax(ly, __shfl_xor_sync(0xffffffffu, ly, o));
        lz = fmax(lz, __shfl_xor_sync(0xffffffffu, lz, o));
    }
    __shared__ double red[3][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        red[0][warp] = lx;
        red[1][warp] = ly;
        red[2][warp] = lz;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) {
            lx = fmax(lx, red[0][i]);
            ly = fmax(ly, red[1][i]);
            lz = fmax(lz, red[2][i]);
        }
        atomic_max_nonneg(&bd.eig[0], lx);
        atomic_max_nonneg(&bd.eig[1], ly);
        atomic_max_nonneg(&bd.eig[2], lz);
    }
}

}  // namespace nuc3d
