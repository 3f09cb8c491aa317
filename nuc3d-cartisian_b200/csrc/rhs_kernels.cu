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
template <typename B>
struct InvTile<1, B> {  // sweep along y: tile = TL columns (i) x TC cells (y)
    static constexpr int TL = 32, TC = 16;
};
template <typename B>
struct InvTile<2, B> {
    static constexpr int TL = 32, TC = 16;
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

// ------------------------------------------------------------ k_visc_flux --
// solveGrads + solveViscousFlux (NaiverStokes3d.cpp:87-303): CD6 gradients of
// u, v, w, T (differences in FP64), stresses and heat flux in the bulk type.
template <typename B>
__global__ void __launch_bounds__(256) k_visc_flux(BoxParams bp, PrimView w, BView9<B> vf) {
    const int nx = bp.n[0], ny = bp.n[1], nz = bp.n[2];
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < bp.N;
         n += (long long)gridDim.x * blockDim.x) {
        int i = (int)(n % nx);
        long long rest = n / nx;
        int j = (int)(rest % ny);
        int k = (int)(rest / ny);
        long long base_x = n - i, base_y = i + (long long)nx * ny * k, base_z = i + (long long)nx * j;
        B g[4][3];
        const int src[4] = {0, 1, 2, 5};  // u, v, w, T
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const double *f = w.w[src[s]];
            // along x
            {
                double d1 = f[base_x + wrap(i + 1, nx)] - f[base_x + wrap(i - 1, nx)];
                double d2 = f[base_x + wrap(i + 2, nx)] - f[base_x + wrap(i - 2, nx)];
                double d3 = f[base_x + wrap(i + 3, nx)] - f[base_x + wrap(i - 3, nx)];
                g[s][0] = B((K::CD3 * d3 + K::CD2 * d2 + K::CD1 * d1) * bp.inv_d[0]);
            }
            {
                long long sy = nx;
                double d1 = f[base_y + sy * wrap(j + 1, ny)] - f[base_y + sy * wrap(j - 1, ny)];
                double d2 = f[base_y + sy * wrap(j + 2, ny)] - f[base_y + sy * wrap(j - 2, ny)];
                double d3 = f[base_y + sy * wrap(j + 3, ny)] - f[base_y + sy * wrap(j - 3, ny)];
                g[s][1] = B((K::CD3 * d3 + K::CD2 * d2 + K::CD1 * d1) * bp.inv_d[1]);
            }
            {
                long long sz = (long long)nx * ny;
                double d1 = f[base_z + sz * wrap(k + 1, nz)] - f[base_z + sz * wrap(k - 1, nz)];
                double d2 = f[base_z + sz * wrap(k + 2, nz)] - f[base_z + sz * wrap(k - 2, nz)];
                double d3 = f[base_z + sz * wrap(k + 3, nz)] - f[base_z + sz * wrap(k - 3, nz)];
                g[s][2] = B((K::CD3 * d3 + K::CD2 * d2 + K::CD1 * d1) * bp.inv_d[2]);
            }
        }
        B ux = g[0][0], uy = g[0][1], uz = g[0][2];
        B vx = g[1][0], vy = g[1][1], vz = g[1][2];
        B wx = g[2][0], wy = g[2][1], wz = g[2][2];
        B tx = g[3][0], ty = g[3][1], tz = g[3][2];
        B grad = ux + vy + wz;
        B miu0, coeff0;
        viscosity<B>(bp, B(w.w[5][n]), miu0, coeff0);
        const B c23 = B(2.0 / 3.0);
        const bool od = (bp.quirks & QK_OFFDIAG_DIV) != 0;
        B dv = od ? c23 * grad : B(0);
        B t_xx = miu0 * (B(2) * ux - c23 * grad);
        B t_xy = miu0 * (uy + vx - dv);
        B t_xz = miu0 * (uz + wx - dv);
        B t_yy = miu0 * (B(2) * vy - c23 * grad);
        B t_yz = miu0 * (vz + wy - dv);
        B t_zz = miu0 * (B(2) * wz - c23 * grad);
        B u = B(w.w[0][n]), v = B(w.w[1][n]), ww = B(w.w[2][n]);
        vf.f[0][n] = t_xx;
        vf.f[1][n] = t_xy;
        vf.f[2][n] = t_xz;
        vf.f[3][n] = t_yy;
        vf.f[4][n] = t_yz;
        vf.f[5][n] = t_zz;
        vf.f[6][n] = u * t_xx + v * t_xy + ww * t_xz + coeff0 * tx;
        vf.f[7][n] = u * t_xy + v * t_yy + ww * t_yz + coeff0 * ty;
        vf.f[8][n] = u * t_xz + v * t_yz + ww * t_zz + coeff0 * tz;
    }
}

// --------------------------------------------------------------- k_update --
// setDerivativesVis (NaiverStokes3d.cpp:305-369): CD6 of the viscous fluxes,
// RHS = inviscid - viscous (:385-499), then the TVD-RK3 stage
// (TVD-RK3.cpp:76-196, dQ/dt = -RHS) in FP64, plus the residual sum of
// PDEData3d::setRES (PDEData3d.cpp:178-213) on the last stage and a finite
// check of the new state.
template <typename B>
__global__ void __launch_bounds__(256)
    k_update(BoxParams bp, BView<B> r, BView9<B> vf, StateView un, StateView uin,
             StateViewMut uout, int stage, const StepScalars *sc, double *res_acc,
             unsigned *flags) {
    const int nx = bp.n[0], ny = bp.n[1], nz = bp.n[2];
    const double dt = sc->dt;
    double res = 0.0;
    bool bad = false;
    const bool vis = bp.navier_stokes != 0;
    for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < bp.N;
         n += (long long)gridDim.x * blockDim.x) {
        B R[5];
#pragma unroll
        for (int e = 0; e < 5; ++e) R[e] = r.f[e][n];
        if (vis) {
            int i = (int)(n % nx);
            long long rest = n / nx;
            int j = (int)(rest % ny);
            int k = (int)(rest / ny);
            long long bx = n - i, by = i + (long long)nx * ny * k, bz = i + (long long)nx * j;
            long long sy = nx, sz = (long long)nx * ny;
            const B ix = B(bp.inv_d[0]), iy = B(bp.inv_d[1]), iz = B(bp.inv_d[2]);
            // x: tau_xx, tau_xy, tau_xz, E_x ; y: tau_xy, tau_yy, tau_yz, E_y ;
            // z: tau_xz, tau_yz, tau_zz, E_z
            const int cx[4] = {0, 1, 2, 6}, cy[4] = {1, 3, 4, 7}, cz[4] = {2, 4, 5, 8};
            B dfx[4], dfy[4], dfz[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const B *f = vf.f[cx[e]];
                dfx[e] = cd6<B>(f[bx + wrap(i - 3, nx)], f[bx + wrap(i - 2, nx)],
                                f[bx + wrap(i - 1, nx)], f[bx + wrap(i + 1, nx)],
                                f[bx + wrap(i + 2, nx)], f[bx + wrap(i + 3, nx)], ix);
                f = vf.f[cy[e]];
                dfy[e] = cd6<B>(f[by + sy * wrap(j - 3, ny)], f[by + sy * wrap(j - 2, ny)],
                                f[by + sy * wrap(j - 1, ny)], f[by + sy * wrap(j + 1, ny)],
                                f[by + sy * wrap(j + 2, ny)], f[by + sy * wrap(j + 3, ny)], iy);
                f = vf.f[cz[e]];
                dfz[e] = cd6<B>(f[bz + sz * wrap(k - 3, nz)], f[bz + sz * wrap(k - 2, nz)],
                                f[bz + sz * wrap(k - 1, nz)], f[bz + sz * wrap(k + 1, nz)],
                                f[bz + sz * wrap(k + 2, nz)], f[bz + sz * wrap(k + 3, nz)], iz);
            }
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                B t = R[1 + e];
                t -= dfx[e];
                t -= dfy[e];
                t -= dfz[e];
                R[1 + e] = t;
            }
        }
        if (stage < 0) {  // RHS only (nuc3d_rhs)
#pragma unroll
            for (int e = 0; e < 5; ++e) uout.q[e][n] = double(R[e]);
            continue;
        }
#pragma unroll
        for (int e = 0; e < 5; ++e) {
            double rhs = -double(R[e]);
            double u_n = un.q[e][n];
            double out;
            if (stage == 0) {
                out = 1.0 * uin.q[e][n] + 1.0 * rhs * dt;
            } else if (stage == 1) {
                out = 0.75 * u_n + 0.25 * (rhs * dt + uin.q[e][n]);
            } else {
                out = (1.0 / 3.0) * u_n + (2.0 / 3.0) * (rhs * dt + uin.q[e][n]);
                double dd = out - u_n;
                res += dd * dd;
            }
            bad |= !isfinite(out);
            uout.q[e][n] = out;
        }
    }
    if (bad) atomicOr(flags, 1u);
    if (stage != 2) return;
    for (int o = 16; o > 0; o >>= 1) res += __shfl_xor_sync(0xffffffffu, res, o);
    __shared__ double red[8];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) red[warp] = res;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < (int)(blockDim.x >> 5); ++i) res += red[i];
        atomicAdd(res_acc, res);
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

template <typename B>
cudaError_t launch_visc_flux(const BoxParams &bp, PrimView w, BView9<B> vf, int sms,
                             cudaStream_t st) {
    k_visc_flux<B><<<grid_for(bp.N, sms), 256, 0, st>>>(bp, w, vf);
    return cudaGetLastError();
}

template <typename B>
cudaError_t launch_update(const BoxParams &bp, BView<B> r, BView9<B> vf, StateView un,
                          StateView uin, StateViewMut uout, int stage, const StepScalars *sc,
                          double *res_acc, unsigned *flags, int sms, cudaStream_t st) {
    k_update<B><<<grid_for(bp.N, sms), 256, 0, st>>>(bp, r, vf, un, uin, uout, stage, sc,
                                                     res_acc, flags);
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
template cudaError_t launch_visc_flux<double>(const BoxParams &, PrimView, BView9<double>, int,
                                              cudaStream_t);
template cudaError_t launch_visc_flux<float>(const BoxParams &, PrimView, BView9<float>, int,
                                             cudaStream_t);
template cudaError_t launch_update<double>(const BoxParams &, BView<double>, BView9<double>,
                                           StateView, StateView, StateViewMut, int,
                                           const StepScalars *, double *, unsigned *, int,
                                           cudaStream_t);
template cudaError_t launch_update<float>(const BoxParams &, BView<float>, BView9<float>,
                                          StateView, StateView, StateViewMut, int,
                                          const StepScalars *, double *, unsigned *, int,
                                          cudaStream_t);

}  // namespace nuc3d
