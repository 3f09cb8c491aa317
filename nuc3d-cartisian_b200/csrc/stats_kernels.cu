// Turbulence statistics of a box's current state on the device, FP64:
// postproc::solveQ (postproc.cpp:736-930) — the velocity-gradient averages,
// vorticity, enstrophy, Q, helicity and kinetic energy of enstrophy.dat and
// the sums behind turb_para.dat — plus the viscous dissipation
// <mu (|omega|^2 + 4/3 (div u)^2)>, which the reference does not compute.
// Gradients are the primitives' derivatives by each direction's differential
// scheme (cd6, cd2 or cd8) with the periodic wrap (the operator's
// differential scheme on one rank, postproc.cpp:2111-2124, :2285-2297).
//
// One launch of a fixed grid accumulates per-block partial sums in a fixed
// order; a one-block launch adds the partials in a fixed order, so the
// result does not depend on what else runs.
#include "rhs_kernels.h"
#include "stats_kernels.h"

namespace nuc3d {

namespace {

constexpr int kThreads = 256;

template <int NV>
__device__ void block_sum(double (&v)[NV], double *out) {
    __shared__ double red[NV][kThreads / 32];
    for (int i = 0; i < NV; ++i) {
        double s = v[i];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[i][threadIdx.x >> 5] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NV; i += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) s += red[i][w];
        out[i] = s;
    }
}

__global__ void __launch_bounds__(kThreads) k_stats(BoxDev b, double *partials) {
    const BoxParams &p = b.p;
    const double *rho = fieldU(b, 0, 0);
    const double *u = fieldW(b, 0), *v = fieldW(b, 1), *w = fieldW(b, 2);
    const double *cs = fieldW(b, 4), *T = fieldW(b, 5);
    const double s_nd = p.tref_nd;
    double acc[kStatsSums];
#pragma unroll
    for (int s = 0; s < kStatsSums; ++s) acc[s] = 0.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < p.N;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % p.n[0]);
        const int j = (int)((c / p.n[0]) % p.n[1]);
        const int k = (int)(c / ((long long)p.n[0] * p.n[1]));
        const double u0 = u[c], u1 = v[c], u2 = w[c];
        const double ux = diff_at(u, p, i, j, k, 0), uy = diff_at(u, p, i, j, k, 1),
                     uz = diff_at(u, p, i, j, k, 2);
        const double vx = diff_at(v, p, i, j, k, 0), vy = diff_at(v, p, i, j, k, 1),
                     vz = diff_at(v, p, i, j, k, 2);
        const double wx = diff_at(w, p, i, j, k, 0), wy = diff_at(w, p, i, j, k, 1),
                     wz = diff_at(w, p, i, j, k, 2);
        // postproc.cpp:812-853
        const double w0 = wy - vz, w1 = uz - wx, w2 = vx - uy;
        const double q0 = ux * vy + ux * wz + vy * wz - uy * vx - uz * wx - vz * wy;
        const double om2 = w0 * w0 + w1 * w1 + w2 * w2;
        acc[0] += ux;
        acc[1] += uy;
        acc[2] += uz;
        acc[3] += vx;
        acc[4] += vy;
        acc[5] += vz;
        acc[6] += wx;
        acc[7] += wy;
        acc[8] += wz;
        acc[9] += w0;
        acc[10] += w1;
        acc[11] += w2;
        acc[12] += om2 * 0.5;
        acc[13] += q0;
        acc[14] += w0 * u0 + w1 * u1 + w2 * u2;
        acc[15] += 0.5 * rho[c] * (u0 * u0 + u1 * u1 + u2 * u2);
        acc[16] += (u0 * u0 + u1 * u1 + u2 * u2) / 3.0;
        acc[17] += (ux * ux + vy * vy + wz * wz) / 3.0;
        acc[18] += (pow(ux, 3.0) + pow(vy, 3.0) + pow(wz, 3.0)) / 3.0;
        acc[19] += cs[c];
        const double Tc = T[c];
        acc[20] += (1.0 + s_nd) / (Tc + s_nd) * pow(Tc, 1.5);
        acc[21] += rho[c];
        double miu, coeff;
        viscosity<double>(p, Tc, miu, coeff);
        const double th = ux + vy + wz;
        acc[22] += miu * (om2 + 4.0 / 3.0 * th * th);
    }
    block_sum<kStatsSums>(acc, partials + (size_t)blockIdx.x * kStatsSums);
}

__global__ void __launch_bounds__(kThreads) k_stats_reduce(const double *partials, int nblocks,
                                                             double *out) {
    double acc[kStatsSums];
#pragma unroll
    for (int s = 0; s < kStatsSums; ++s) acc[s] = 0.0;
    for (int bl = threadIdx.x; bl < nblocks; bl += blockDim.x)
        for (int s = 0; s < kStatsSums; ++s) acc[s] += partials[(size_t)bl * kStatsSums + s];
    block_sum<kStatsSums>(acc, out);
}

}  // namespace

cudaError_t launch_stats(const BoxDev &b, double *scratch, cudaStream_t st) {
    k_stats<<<kStatsBlocks, kThreads, 0, st>>>(b, scratch + kStatsSums);
    k_stats_reduce<<<1, kThreads, 0, st>>>(scratch + kStatsSums, kStatsBlocks, scratch);
    return cudaGetLastError();
}

void stats_finish(const BoxParams &p, const double *sums, double *out) {
    // postproc.cpp:855-876; the field averages as MPICommunicator.cpp:161-185
    const double NN = (double)p.N;
    for (int s = 0; s < 16; ++s) out[s] = sums[s] / NN;
    const double u_rms_aver = sums[16] / NN, div_aver = sums[17] / NN, skew3 = sums[18] / NN;
    const double skew2 = div_aver, alpha_aver = sums[19] / NN, miu_aver = sums[20] / NN;
    const double rho_bar = sums[21] / NN;
    const double skew = skew3 / std::pow(skew2, 1.5);
    const double lambda = std::sqrt(u_rms_aver / div_aver);
    const double re_lambda = std::sqrt(u_rms_aver) * lambda * rho_bar / miu_aver * p.reynolds;
    const double tau_t = lambda / std::sqrt(u_rms_aver);
    out[16] = std::sqrt(u_rms_aver);
    out[17] = std::sqrt(u_rms_aver * 3.0) / alpha_aver;
    out[18] = std::sqrt(div_aver);
    out[19] = miu_aver;
    out[20] = re_lambda;
    out[21] = lambda;
    out[22] = rho_bar;
    out[23] = tau_t;
    out[24] = skew;
    out[25] = sums[22] / NN;
}

}  // namespace nuc3d
