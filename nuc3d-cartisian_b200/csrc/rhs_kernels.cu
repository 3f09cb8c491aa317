// Whole-box RHS + TVD-RK3 stage kernels for one periodic box.
//
// One stage = k_prim -> [k_visc_flux] -> k_inviscid<x> -> k_inviscid<y> ->
// k_inviscid<z> -> k_update.  The reference's per-direction rotated copies,
// halo buffers and MPI self-messages (euler3d.cpp:307-387,
// NaiverStokes3d.cpp:87-369, MPICommunicator.cpp:81-132) become periodic
// index wraps inside the tile loads.
#include "nuc3d_device.cuh"
#include "rhs_kernels.h"

namespace nuc3d {

// ----------------------------------------------------------------- k_prim --
// physicsModel::con2prim (physicsModel.cpp:324-356), FP64, plus the running
// maxEigen of RiemannLF (physicsModel.cpp:546-547, 600-601, 653-654).
__global__ void __launch_bounds__(256) k_prim(BoxParams bp, StateView q, PrimView w,
                                              double *eig, int want_eig) {
    double lx = 0.0, ly = 0.0, lz = 0.0;
    const double gamma = bp.gamma, Mach = bp.mach;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < bp.N;
         n += (long long)gridDim.x * blockDim.x) {
        double rho = q.q[0][n];
        double u = q.q[1][n] / rho;
        double v = q.q[2][n] / rho;
        double ww = q.q[3][n] / rho;
        double E = q.q[4][n];
        double p = (E - 0.5 * rho * (u * u + v * v + ww * ww)) * (gamma - 1.0);
        if (bp.quirks & QK_FABS_PRESSURE) p = fabs(p);
        double c = sqrt(gamma * p / rho);
        double T = gamma * Mach * Mach * p / rho;
        w.w[0][n] = u;
        w.w[1][n] = v;
        w.w[2][n] = ww;
        w.w[3][n] = p;
        w.w[4][n] = c;
        w.w[5][n] = T;
        lx = fmax(fabs(u) + c, lx);
        ly = fmax(fabs(v) + c, ly);
        lz = fmax(fabs(ww) + c, lz);
    }
    if (!want_eig) return;
    if (bp.quirks & QK_ZETA_EIGEN) {  // z loop writes MaxEigen_eta; zeta stays 0
        ly = fmax(lz, ly);
        lz = 0.0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        lx = fmax(lx, __shfl_xor_sync(0xffffffffu, lx, o));
        ly = fmax(ly, __shfl_xor_sync(0xffffffffu, ly, o));
        lz = fmax(lz, __shfl_xor_sync(0xffffffffu, lz, o));
    }
    __shared__ double red[3][8];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
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
        atomic_max_nonneg(&eig[0], lx);
        atomic_max_nonneg(&eig[1], ly);
        atomic_max_nonneg(&eig[2], lz);
    }
}

// -------------------------------------------------------------------- k_dt --
// EulerData3D::getDt (euler3d.cpp:459-466) and PDEData3d::solve's
// dt_global = dt_local * cfl (PDEData3d.cpp:161-165).  One thread.
__global__ void k_dt(BoxParams bp, const double *eig, StepScalars *sc, int step) {
    double dt_xi = bp.d[0] / eig[0];
    double dt_eta = bp.d[1] / eig[1];
    double dt_zeta = bp.d[2] / eig[2];
    double dt_local = 1.0 / (1.0 / dt_xi + 1.0 / dt_eta + 1.0 / dt_zeta);
    sc->dt_local = dt_local;
    sc->dt = dt_local * bp.cfl;
    if (step >= 0) sc->dt_hist[step] = sc->dt;
}

// -------------------------------------------------------------- k_inviscid --
// Tile geometry of the directional sweep kernel.
template <int DIR, typename B>
struct InvTile;
template <typename B>
struct InvTile<0, B> {  // sweep along x: tile = TL rows (j) x TC cells (x)
    static constexpr int TL = 8, TC = 32;
};
// sweep along y / z: tile = TL columns (i) x TC cells along the sweep.  TL
// columns of B make one full 128-byte row per load; FP64 uses 16 columns so
// that four to five blocks fit per SM.
template <typename B>
struct InvTile<1, B> {
    static constexpr int TL = 128 / sizeof(B), TC = 16;
};
template <typename B>
struct InvTile<2, B> {
    static constexpr int TL = 128 / sizeof(B), TC = 16;
};

template <int DIR, typename B>
struct InvGeom {
    static constexpr int TL = InvTile<DIR, B>::TL, TC = InvTile<DIR, B>::TC;
    static constexpr int NF = TC + 6;  // cells staged (3-cell halo each side)
    static constexpr int NH = TC + 1;  // faces
    static constexpr int NT = TL * NH; // threads: one face per thread
    // shared-memory index: thread-fast index is the position for DIR 0 and
    // the line for DIR 1/2, so neighbouring threads touch neighbouring words
    __device__ static int sf(int v, int l, int pc) {
        return DIR == 0 ? (v * TL + l) * NF + pc : (v * NF + pc) * TL + l;
    }
    __device__ static int sh(int e, int l, int m) {
        return DIR == 0 ? (e * TL + l) * NH + m : (e * NH + m) * TL + l;
    }
    __device__ static void item(int t, int span, int &l, int &p) {
        if (DIR == 0) {
            l = t / span;
            p = t - l * span;
        } else {
            l = t % TL;
            p = t / TL;
        }
    }
};

// Inviscid flux derivative along DIR for all 5 equations (euler3d.cpp:307-387
// + combineFluxLR :23-56 + setDerivatives*Inv :143-253), with the
// Lax-Friedrichs split (physicsModel.cpp:546-565) done while staging.
//   accumulate = 0: r = dF/dx ; 1: r += dG/dy (rhs order of
//   NaiverStokes3d.cpp:396-446).
// Mixed precision (B = float): the split fluxes are formed in FP64 and each
// line's value at the tile's first interior cell is subtracted before
// rounding to FP32.  WENO5 commutes with adding a constant and the constant
// cancels in the face difference, so this only removes rounding error.
template <int SCHEME, int DIR, typename B>
__global__ void __launch_bounds__(InvGeom<DIR, B>::NT)
    k_inviscid(BoxParams bp, StateView q, PrimView w, BView<B> r, int accumulate) {
    using G = InvGeom<DIR, B>;
    constexpr int TL = G::TL, TC = G::TC, NF = G::NF, NH = G::NH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    B *sF = reinterpret_cast<B *>(smem_raw);      // [10][..] split fluxes (+ e, then - e)
    B *sH = sF + 10 * TL * NF;                     // [5][..] face fluxes F^+ + F^-
    __shared__ double sRef[10][TL];

    const int n = bp.n[DIR];
    int l0, c0, fixed;  // first line, first cell of the chunk, the third index
    if (DIR == 0) {
        c0 = blockIdx.x * TC;
        l0 = blockIdx.y * TL;
        fixed = blockIdx.z;
    } else if (DIR == 1) {
        l0 = blockIdx.x * TL;
        c0 = blockIdx.y * TC;
        fixed = blockIdx.z;
    } else {
        l0 = blockIdx.x * TL;
        fixed = blockIdx.y;
        c0 = blockIdx.z * TC;
    }
    const int nl = DIR == 0 ? bp.n[1] : bp.n[0];  // extent of the line index
    auto gidx = [&](int l, int pos) -> long long {
        int a = l0 + l;
        if (DIR == 0) return pos + bp.stride[1] * (a + (long long)bp.n[1] * fixed);
        if (DIR == 1) return a + bp.stride[1] * (pos + (long long)bp.n[1] * fixed);
        return a + bp.n[0] * (long long)fixed + bp.stride[2] * pos;
    };
    auto split = [&](long long g, double Fp[5], double Fm[5]) {
        double Q[5] = {q.q[0][g], q.q[1][g], q.q[2][g], q.q[3][g], q.q[4][g]};
        double un = w.w[DIR][g], p = w.w[3][g], c = w.w[4][g];
        double lam = fabs(un) + c;
        double f[5];
#pragma unroll
        for (int e = 0; e < 4; ++e) f[e] = un * Q[e];
        f[1 + DIR] = un * Q[1 + DIR] + p;
        f[4] = un * (Q[4] + p);
#pragma unroll
        for (int e = 0; e < 5; ++e) {
            Fp[e] = 0.5 * (f[e] + lam * Q[e]);
            Fm[e] = 0.5 * (f[e] - lam * Q[e]);
        }
    };
    const bool mixed = sizeof(B) == sizeof(float);
    if (mixed) {  // per-line reference values (cell c0, always inside the box)
        if (threadIdx.x < TL) {
            int l = threadIdx.x;
            double Fp[5], Fm[5];
            if (l0 + l < nl) {
                split(gidx(l, c0), Fp, Fm);
            } else {
#pragma unroll
                for (int e = 0; e < 5; ++e) Fp[e] = Fm[e] = 0.0;
            }
#pragma unroll
            for (int e = 0; e < 5; ++e) {
                sRef[e][l] = Fp[e];
                sRef[5 + e][l] = Fm[e];
            }
        }
        __syncthreads();
    }
    // phase 1: stage the split fluxes of cells c0-3 .. c0+TC+2
    for (int t = threadIdx.x; t < TL * NF; t += blockDim.x) {
        int l, pc;
        G::item(t, NF, l, pc);
        double Fp[5], Fm[5];
        if (l0 + l < nl) {
            int pos = ((c0 - 3 + pc) % n + n) % n;
            split(gidx(l, pos), Fp, Fm);
        } else {
#pragma unroll
            for (int e = 0; e < 5; ++e) Fp[e] = Fm[e] = 0.0;
        }
#pragma unroll
        for (int e = 0; e < 5; ++e) {
            if (mixed) {
                sF[G::sf(e, l, pc)] = B(Fp[e] - sRef[e][l]);
                sF[G::sf(5 + e, l, pc)] = B(Fm[e] - sRef[5 + e][l]);
            } else {
                sF[G::sf(e, l, pc)] = B(Fp[e]);
                sF[G::sf(5 + e, l, pc)] = B(Fm[e]);
            }
        }
    }
    __syncthreads();
    // phase 2: faces c0 .. c0+TC (face m lies between cells m-1 and m)
    const bool zq = SCHEME == SCHEME_Z && (bp.quirks & QK_WENOZ_BETA2);
    for (int t = threadIdx.x; t < TL * NH; t += blockDim.x) {
        int l, m;
        G::item(t, NH, l, m);
        int gm = c0 + m;
        if (gm > n) continue;
        // weno5z.cpp:80 applies on the inner faces 3..n-3 only
        bool quirk = zq && gm >= 3 && gm <= n - 3;
#pragma unroll 1
        for (int e = 0; e < 5; ++e) {
            // '+': cells gm-3..gm+1 -> pc m..m+4 ; '-': cells gm+2..gm-2 -> pc m+5..m+1
            B fp = weno5_face<SCHEME, B>(sF[G::sf(e, l, m)], sF[G::sf(e, l, m + 1)],
                                         sF[G::sf(e, l, m + 2)], sF[G::sf(e, l, m + 3)],
                                         sF[G::sf(e, l, m + 4)], quirk);
            B fm = weno5_face<SCHEME, B>(sF[G::sf(5 + e, l, m + 5)], sF[G::sf(5 + e, l, m + 4)],
                                         sF[G::sf(5 + e, l, m + 3)], sF[G::sf(5 + e, l, m + 2)],
                                         sF[G::sf(5 + e, l, m + 1)], false);
            sH[G::sh(e, l, m)] = fp + fm;
        }
    }
    __syncthreads();
    // phase 3: dF/dx(cell) = (F^[m+1] - F^[m]) / delta
    const B inv_d = B(bp.inv_d[DIR]);
    for (int t = threadIdx.x; t < TL * TC; t += blockDim.x) {
        int l, m;
        G::item(t, TC, l, m);
        int gc = c0 + m;
        if (gc >= n || l0 + l >= nl) continue;
        long long g = gidx(l, gc);
#pragma unroll
        for (int e = 0; e < 5; ++e) {
            B dfe = (sH[G::sh(e, l, m + 1)] - sH[G::sh(e, l, m)]) * inv_d;
            if (accumulate)
                r.f[e][g] += dfe;
            else
                r.f[e][g] = dfe;
        }
    }
}

// k_residual_final: residual = sqrt(sum / (5 N)) / dt (PDEData3d.cpp:212)
__global__ void k_residual(BoxParams bp, StepScalars *sc, double *res_acc, int step) {
    double r = sqrt(*res_acc / (double)(bp.N * 5)) / sc->dt;
    if (step >= 0) sc->res_hist[step] = r;
    sc->time += sc->dt;
    *res_acc = 0.0;
}

// --------------------------------------------------------------- launches --
static int grid_for(long long N, int sms) {
    long long want = (N + 255) / 256;
    long long cap = (long long)sms * 8;
    return (int)(want < cap ? want : cap);
}

template <typename B>
static size_t inv_smem(int dir) {
    auto f = [](int TL, int TC) { return sizeof(B) * (size_t)(10 * TL * (TC + 6) + 5 * TL * (TC + 1)); };
    if (dir == 0) return f(InvTile<0, B>::TL, InvTile<0, B>::TC);
    if (dir == 1) return f(InvTile<1, B>::TL, InvTile<1, B>::TC);
    return f(InvTile<2, B>::TL, InvTile<2, B>::TC);
}

template <int SCHEME, int DIR, typename B>
static cudaError_t launch_inviscid_t(const BoxParams &bp, StateView q, PrimView w, BView<B> r,
                                     int accumulate, cudaStream_t st) {
    using G = InvGeom<DIR, B>;
    size_t sm = inv_smem<B>(DIR);
    auto kern = k_inviscid<SCHEME, DIR, B>;
    static bool attr_set = false;  // per template instance
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    dim3 grid;
    if (DIR == 0)
        grid = dim3((bp.n[0] + G::TC - 1) / G::TC, (bp.n[1] + G::TL - 1) / G::TL, bp.n[2]);
    else if (DIR == 1)
        grid = dim3((bp.n[0] + G::TL - 1) / G::TL, (bp.n[1] + G::TC - 1) / G::TC, bp.n[2]);
    else
        grid = dim3((bp.n[0] + G::TL - 1) / G::TL, bp.n[1], (bp.n[2] + G::TC - 1) / G::TC);
    kern<<<grid, G::NT, sm, st>>>(bp, q, w, r, accumulate);
    return cudaGetLastError();
}

template <typename B>
cudaError_t launch_inviscid(const BoxParams &bp, int dir, StateView q, PrimView w, BView<B> r,
                            int accumulate, cudaStream_t st) {
    int s = bp.scheme[dir];
    if (s == SCHEME_JS) {
        if (dir == 0) return launch_inviscid_t<SCHEME_JS, 0, B>(bp, q, w, r, accumulate, st);
        if (dir == 1) return launch_inviscid_t<SCHEME_JS, 1, B>(bp, q, w, r, accumulate, st);
        return launch_inviscid_t<SCHEME_JS, 2, B>(bp, q, w, r, accumulate, st);
    }
    if (s == SCHEME_Z) {
        if (dir == 0) return launch_inviscid_t<SCHEME_Z, 0, B>(bp, q, w, r, accumulate, st);
        if (dir == 1) return launch_inviscid_t<SCHEME_Z, 1, B>(bp, q, w, r, accumulate, st);
        return launch_inviscid_t<SCHEME_Z, 2, B>(bp, q, w, r, accumulate, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_prim(const BoxParams &bp, StateView q, PrimView w, double *eig, int want_eig,
                        int sms, cudaStream_t st) {
    k_prim<<<grid_for(bp.N, sms), 256, 0, st>>>(bp, q, w, eig, want_eig);
    return cudaGetLastError();
}

cudaError_t launch_dt(const BoxParams &bp, const double *eig, StepScalars *sc, int step,
                      cudaStream_t st) {
    k_dt<<<1, 1, 0, st>>>(bp, eig, sc, step);
    return cudaGetLastError();
}

cudaError_t launch_residual(const BoxParams &bp, StepScalars *sc, double *res_acc, int step,
                            cudaStream_t st) {
    k_residual<<<1, 1, 0, st>>>(bp, sc, res_acc, step);
    return cudaGetLastError();
}

template cudaError_t launch_inviscid<double>(const BoxParams &, int, StateView, PrimView,
                                             BView<double>, int, cudaStream_t);
template cudaError_t launch_inviscid<float>(const BoxParams &, int, StateView, PrimView,
                                            BView<float>, int, cudaStream_t);
}  // namespace nuc3d
