// 2.5-D blocked stencil kernels of the viscous part and the RK update.
//
// A block owns a 32 x 8 column tile of the box and marches a chunk of
// `depth` planes along z (the pencil depth, a launch argument the engine's
// autotuner picks).  For each plane it stages the tile plus the x/y halo in
// shared memory (the x- and y-direction stencils read it there) while every
// thread keeps a (2R+1)-deep register queue of its own column for the
// z-direction stencil, so each value is fetched from L2/HBM about once per
// plane instead of once per stencil tap.
//
// R is the stencil reach.  R = 3: boxes whose three directions use cd6 (the
// CD6 stencil written out).  R = 4: every other box; each direction's
// differential scheme (cd2, cd6 or cd8) is its coefficients of
// f(i+m) - f(i-m), m = 1..4 (BoxParams::vcoef, zero beyond its reach).
#include "nuc3d_device.cuh"
#include "rhs_kernels.h"

namespace nuc3d {

namespace {

constexpr int TX = kT25X, TY = kT25Y;

// a TMA tensor map as the kernels see it: 128 opaque, 64-byte aligned bytes
// (the host encodes CUtensorMap values into the box's allocation)
struct alignas(64) CUtensorMapLike {
    unsigned long long opaque[16];
};

// Asynchronous global->shared copy of one element (cp.async, L1-allocating),
// so a plane's halo tile streams in while the previous plane is computed.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *smem, const T *gmem) {
    unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(gmem),
                 "n"(sizeof(T)));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

// ---- TMA (cp.async.bulk.tensor) loads completed on an mbarrier ----
__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// waits for the completion of phase `parity` of the barrier for at most
// ~2^31 clock cycles (about a second); false on timeout
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
    const long long t0 = clock64();
    while (true) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > (1ll << 31)) return false;
    }
}
// one 3-D tile of a tensor map (coordinates x, y, z in elements) into shared
// memory, completing on the barrier
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, int x, int y, int z,
                                            unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ int pmod(int c, int n) {
    int r = c % n;
    return r < 0 ? r + n : r;
}
// c mod n for c in [-n, 2n) (a halo index of at most one period outside the
// box): a compare and an add instead of a division
__device__ __forceinline__ int wrap1(int c, int n) {
    c += c < 0 ? n : 0;
    return c >= n ? c - n : c;
}

__device__ __forceinline__ double cd6d(double m3, double m2, double m1, double p1, double p2,
                                       double p3, double inv) {
    return (K::CD3 * (p3 - m3) + K::CD2 * (p2 - m2) + K::CD1 * (p1 - m1)) * inv;
}

// a direction's differential scheme from the cells at offsets -4..4:
// c[m-1] is its coefficient of f(i+m) - f(i-m)
template <typename T, typename C>
__device__ __forceinline__ T cd_any(T m4, T m3, T m2, T m1, T p1, T p2, T p3, T p4, const C *c,
                                   T inv) {
    return (T(c[3]) * (p4 - m4) + T(c[2]) * (p3 - m3) + T(c[1]) * (p2 - m2) +
            T(c[0]) * (p1 - m1)) *
           inv;
}

}  // namespace

// solveGrads + solveViscousFlux (NaiverStokes3d.cpp:87-303): gradients of
// u, v, w, T by the differential schemes (FP64 differences), stresses and
// heat flux in the bulk type, written as tau_xx, tau_xy, tau_xz, tau_yy,
// tau_yz, tau_zz, E_x, E_y, E_z.
// Work item: (box, x tile, y tile, z chunk of `depth` planes).
template <typename B, int R>
__global__ void __launch_bounds__(TX *TY, 2) k_visc_flux25(const BoxDev *__restrict__ boxes, const WorkItem *__restrict__ items, int depth) {
    // dynamic shared memory (visc_smem_bytes): the two plane tiles with their
    // x/y halo (row pitch TX + 8: column 0 is cell i0 - 4, so that a TMA box
    // starts on a 32-byte boundary), each column's plane k+R (z-queue
    // refill), the tile offsets, two mbarriers
    static_assert(R == 3 || R == 4, "stencil reach");
    static_assert(kViscTmaHaloX == TX + 8 && kViscTmaHaloY == TY + 6, "TMA halo box");
    static_assert(kViscTmaTileX == TX && kViscTmaTileY == TY, "TMA tile box");
    constexpr int QD = 2 * R + 1;                   // z-queue depth
    constexpr int RY = TY + 2 * R, RX = TX + 2 * R;  // halo tile rows, halo columns
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // TMA destinations must start on 128-byte boundaries: the layout starts
    // at the first such boundary of the window (128 bytes are reserved)
    unsigned char *const sbase = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
    constexpr int PX = TX + 8;
    auto sP = reinterpret_cast<double (*)[4][RY][PX]>(sbase);
    auto sZ = reinterpret_cast<double (*)[4][TX * TY]>(sbase + sizeof(double) * 2 * 4 * RY * PX);
    int *sOff = reinterpret_cast<int *>(sbase + sizeof(double) * 2 * 4 * (RY * PX + TX * TY));
    auto mbar = reinterpret_cast<unsigned long long *>(
        sbase + sizeof(double) * 2 * 4 * (RY * PX + TX * TY) + 16 * (RY * RX * 4 / 16 + 1));
    const WorkItem it = items[blockIdx.x];
    const BoxDev &bd = boxes[it.box];
    if (!bd.active || !bd.p.navier_stokes) return;
    const BoxParams &bp = bd.p;
    const long long np = bd.np;
    const double *const wbase = fieldW(bd, 0);
    B *const vbase = fieldV<B>(bd, 0);
    const int nx = bp.n[0], ny = bp.n[1], nz = bp.n[2];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = it.a * TX, j0 = it.b * TY, k0 = it.c * depth;
    const int i = i0 + tx, j = j0 + ty;
    const bool active = i < nx && j < ny;
    const long long sz = bp.stride[2];
    const long long col = active ? (long long)i + (long long)nx * j : 0;
    const int src[4] = {0, 1, 2, 5};  // u, v, w, T
    // A CD6 tile (R = 3) whose halo plane lies inside the box (no periodic
    // wrap) loads each plane with TMA: one thread issues 8 tile copies (halo
    // plane and plane k+3 of u, v, w, T) completing on the buffer's mbarrier.
    // Other tiles copy element by element with cp.async through the wrapped
    // offset table.
    const CUtensorMapLike *tm = static_cast<const CUtensorMapLike *>(bd.tmw);
    const bool tma = R == 3 && tm != nullptr && i0 >= 4 && i0 + TX + 4 <= nx && j0 >= 3 &&
                     j0 + TY + 3 <= ny;
    if (tma) {
        if (tid == 0) {
            mbar_init(&mbar[0], 1);
            mbar_init(&mbar[1], 1);
            asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        }
    } else {
        for (int t = tid; t < RY * RX; t += TX * TY) {
            int yy = t / RX, xx = t - yy * RX;
            sOff[t] = pmod(i0 - R + xx, nx) + nx * pmod(j0 - R + yy, ny);
        }
    }
    __syncthreads();
    constexpr unsigned kTmaBytes = 4 * sizeof(double) * ((TY + 6) * PX + TX * TY);
    // plane k's halo tile, and each column's plane k+R for the z-queue: both
    // arrive while plane k-1 is computed
    auto issue = [&](int k, int buf) {
        const int kz = k + R < nz ? k + R : k + R - nz;  // nz >= 8
        if (tma) {
            if (tid == 0) {
                // the buffer's previous contents were read before the block's
                // last barrier; order those reads before the async writes
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                mbar_arrive_expect_tx(&mbar[buf], kTmaBytes);
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    tma_load_3d(&sP[buf][f][0][0], &tm[f], i0 - 4, j0 - 3, k, &mbar[buf]);
                    tma_load_3d(&sZ[buf][f][0], &tm[4 + f], i0, j0, kz, &mbar[buf]);
                }
            }
            return;
        }
        const long long plane = sz * k;
        for (int t = tid; t < RY * RX; t += TX * TY) {
            int yy = t / RX, xx = t - yy * RX;
            long long g = plane + sOff[t];
#pragma unroll
            for (int f = 0; f < 4; ++f)
                cp_async_elem(&sP[buf][f][yy][xx + 4 - R], wbase + src[f] * np + g);
        }
        if (active) {
            const long long g6 = col + sz * kz;
#pragma unroll
            for (int f = 0; f < 4; ++f) cp_async_elem(&sZ[buf][f][tid], wbase + src[f] * np + g6);
        }
    };
    // plane k's buffer is ready: TMA tiles wait on the buffer's barrier (its
    // (k-k0)/2-th completion), cp.async tiles on their own copies and then
    // the block.  False when a TMA wait timed out (the block then stops).
    auto ready = [&](int k, int buf) -> bool {
        if (tma) {
            const bool ok = mbar_wait(&mbar[buf], ((k - k0) >> 1) & 1);
            return !__syncthreads_or(!ok);
        }
        cp_async_wait1();
        __syncthreads();
        return true;
    };
    const int kend = min(k0 + depth, nz);
    issue(k0, 0);
    cp_async_commit();
    double qz[4][QD];
#pragma unroll
    for (int s = 0; s < 2 * R; ++s) {
        long long g = col + sz * pmod(k0 - R + s, nz);
#pragma unroll
        for (int f = 0; f < 4; ++f) qz[f][s] = active ? wbase[src[f] * np + g] : 0.0;
    }
    const double ix = bp.inv_d[0], iy = bp.inv_d[1], iz = bp.inv_d[2];
    const B c23 = B(2.0 / 3.0);
    const bool od = (bp.quirks & QK_OFFDIAG_DIV) != 0;
    const ViscConst<B> vc(bp);
    // The z queue is a ring of QD register slots: plane k+s-R sits in slot
    // (k-k0+s) % QD.  The plane loop is unrolled by QD so that every slot
    // index is a constant and the ring turns without register moves.
    for (int kb = k0; kb < kend; kb += QD) {
#pragma unroll
        for (int u = 0; u < QD; ++u) {
            const int k = kb + u;
            if (k >= kend) break;  // block-uniform
            const int buf = (k - k0) & 1;
            if (k + 1 < kend) issue(k + 1, buf ^ 1);
            cp_async_commit();
            if (!ready(k, buf)) {
                // a TMA wait timed out: report it, give the copies still in
                // flight into both buffers one more bounded wait each, and
                // stop.  The box's state is undefined from here on: the host
                // treats the flag as fatal (NUC3D_ERR_CUDA).
                if (tid == 0) {
                    atomicOr(bd.flags, kFlagWaitTimeout);
                    mbar_wait(&mbar[buf], ((k - k0) >> 1) & 1);
                    if (k + 1 < kend) mbar_wait(&mbar[buf ^ 1], ((k + 1 - k0) >> 1) & 1);
                }
                return;
            }
            // slot of plane k+s-R (kb - k0 is a multiple of QD)
#define QZ(f, s) qz[f][(u + (s)) % QD]
#pragma unroll
            for (int f = 0; f < 4; ++f) QZ(f, 2 * R) = active ? sZ[buf][f][tid] : 0.0;
            if (active) {
                B gr[4][3];
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    const int r = ty + R, c = tx + 4;
                    const double(*P)[PX] = sP[buf][f];
                    if constexpr (R == 3) {
                        gr[f][0] = B(cd6d(P[r][c - 3], P[r][c - 2], P[r][c - 1], P[r][c + 1],
                                          P[r][c + 2], P[r][c + 3], ix));
                        gr[f][1] = B(cd6d(P[r - 3][c], P[r - 2][c], P[r - 1][c], P[r + 1][c],
                                          P[r + 2][c], P[r + 3][c], iy));
                        gr[f][2] = B(cd6d(QZ(f, 0), QZ(f, 1), QZ(f, 2), QZ(f, 4), QZ(f, 5),
                                          QZ(f, 6), iz));
                    } else {
                        gr[f][0] = B(cd_any(P[r][c - 4], P[r][c - 3], P[r][c - 2], P[r][c - 1],
                                            P[r][c + 1], P[r][c + 2], P[r][c + 3], P[r][c + 4],
                                            bp.vcoef[0], ix));
                        gr[f][1] = B(cd_any(P[r - 4][c], P[r - 3][c], P[r - 2][c], P[r - 1][c],
                                            P[r + 1][c], P[r + 2][c], P[r + 3][c], P[r + 4][c],
                                            bp.vcoef[1], iy));
                        gr[f][2] = B(cd_any(QZ(f, 0), QZ(f, 1), QZ(f, 2), QZ(f, 3), QZ(f, 5),
                                            QZ(f, 6), QZ(f, 7), QZ(f, 8), bp.vcoef[2], iz));
                    }
                }
                B ux = gr[0][0], uy = gr[0][1], uz = gr[0][2];
                B vx = gr[1][0], vy = gr[1][1], vz = gr[1][2];
                B wx = gr[2][0], wy = gr[2][1], wz = gr[2][2];
                B tx_ = gr[3][0], ty_ = gr[3][1], tz_ = gr[3][2];
                B grad = ux + vy + wz;
                B miu0, coeff0;
                vc.eval(B(QZ(3, R)), miu0, coeff0);
                B dv = od ? c23 * grad : B(0);
                B t_xx = miu0 * (B(2) * ux - c23 * grad);
                B t_xy = miu0 * (uy + vx - dv);
                B t_xz = miu0 * (uz + wx - dv);
                B t_yy = miu0 * (B(2) * vy - c23 * grad);
                B t_yz = miu0 * (vz + wy - dv);
                B t_zz = miu0 * (B(2) * wz - c23 * grad);
                B uu = B(QZ(0, R)), v = B(QZ(1, R)), ww = B(QZ(2, R));
#undef QZ
                long long g = col + sz * k;
                vbase[0 * np + g] = t_xx;
                vbase[1 * np + g] = t_xy;
                vbase[2 * np + g] = t_xz;
                vbase[3 * np + g] = t_yy;
                vbase[4 * np + g] = t_yz;
                vbase[5 * np + g] = t_zz;
                vbase[6 * np + g] = uu * t_xx + v * t_xy + ww * t_xz + coeff0 * tx_;
                vbase[7 * np + g] = uu * t_xy + v * t_yy + ww * t_yz + coeff0 * ty_;
                vbase[8 * np + g] = uu * t_xz + v * t_yz + ww * t_zz + coeff0 * tz_;
            }
            __syncthreads();
        }
    }
}

// setDerivativesVis (NaiverStokes3d.cpp:305-369): the differential schemes
// of the viscous fluxes,
// RHS = inviscid - viscous in the reference's order (:385-499), then the
// TVD-RK3 stage (TVD-RK3.cpp:76-196, dQ/dt = -RHS) in FP64; on the last stage
// also the residual sum of PDEData3d::setRES (PDEData3d.cpp:178-213).  Every
// new state value passes a finite check.  stage = -1 writes the total RHS.
// Work item: (box, x tile, y tile, z chunk of `depth` planes).  ANYVIS: some box of the batch
// is viscous (sizes the shared tiles); per box the viscous part runs only for
// Navier-Stokes boxes.
template <typename B, bool ANYVIS, int R>
__global__ void __launch_bounds__(TX *TY, 2)
    k_update25(const BoxDev *__restrict__ boxes, const WorkItem *__restrict__ items, int depth,
               StageArgs sa) {
    static_assert(R == 3 || R == 4, "stencil reach");
    constexpr int QD = 2 * R + 1;  // z-queue depth
    // x stencils: tau_xx, tau_xy, tau_xz, E_x; y: tau_xy, tau_yy, tau_yz, E_y;
    // z: tau_xz, tau_yz, tau_zz, E_z
    // x and y halo tiles of the fluxes each stencil direction needs.  (The
    // z-queue refill stays a direct load here: routing it through shared
    // memory as k_visc_flux25 does pushed this kernel into register spills.)
    // R = 3 keeps them in static shared memory; the R = 4 tiles (52 KB in
    // FP64) lie in the dynamic window (update_smem_bytes).
    using XTile = B[2][4][TY][TX + 2 * R];
    using YTile = B[2][4][TY + 2 * R][TX];
    XTile *sXp;
    YTile *sYp;
    if constexpr (R == 3) {
        __shared__ XTile sX3;
        __shared__ YTile sY3;
        sXp = &sX3;
        sYp = &sY3;
    } else {
        extern __shared__ __align__(16) unsigned char smem_dyn[];
        sXp = reinterpret_cast<XTile *>(smem_dyn);
        sYp = reinterpret_cast<YTile *>(smem_dyn + sizeof(XTile));
    }
    XTile &sX = *sXp;
    YTile &sY = *sYp;
    __shared__ double red[TX * TY / 32];
    // periodic wraps of the tile's columns and rows with their R-cell halos
    // (x: i index; y: row offset j nx), resolved once per block.  FP32 only:
    // in the FP64 instance (at its register limit) the table lookups cost
    // register spills that outweigh the remainders they save.
    constexpr bool wrap_table = sizeof(B) == 4;
    __shared__ int sWx[TX + 2 * R], sWy[TY + 2 * R];
    const int cx[4] = {0, 1, 2, 6}, cy[4] = {1, 3, 4, 7}, cz[4] = {2, 4, 5, 8};
    const WorkItem it = items[blockIdx.x];
    const BoxDev &bd = boxes[it.box];
    if (!bd.active) return;
    const BoxParams &bp = bd.p;
    const bool VIS = ANYVIS && bp.navier_stokes;
    const long long np = bd.np;
    const B *const rbase = fieldR<B>(bd, 0);
    const B *const vbase = fieldV<B>(bd, 0);
    const int stage = sa.stage;
    const double *const unb = fieldU(bd, 0, 0);
    const double *const uinb = fieldU(bd, stage < 0 ? 0 : sa.in_slot, 0);
    double *const uoutb = stage < 0 ? nullptr : fieldU(bd, sa.out_slot, 0);
    const StepScalars *sc = bd.sc;
    const int nx = bp.n[0], ny = bp.n[1], nz = bp.n[2];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = it.a * TX, j0 = it.b * TY, k0 = it.c * depth;
    const int i = i0 + tx, j = j0 + ty;
    const bool active = i < nx && j < ny;
    const long long sz = bp.stride[2];
    const long long col = active ? (long long)i + (long long)nx * j : 0;
    const double dt = sc->dt;
    const B ixb = B(bp.inv_d[0]), iyb = B(bp.inv_d[1]), izb = B(bp.inv_d[2]);
    const int kend = min(k0 + depth, nz);
    if constexpr (wrap_table) {
        if (tid < TX + 2 * R) sWx[tid] = pmod(i0 - R + tid, nx);
        if (tid < TY + 2 * R) sWy[tid] = nx * pmod(j0 - R + tid, ny);
        __syncthreads();
    }
    // in-plane offset of tile position (xx, yy) relative to (i0 - R, j0 - R).
    // Active threads read cells i0 - R .. nx + R - 1 (and rows alike); a tile
    // reaching further past the box (a box narrower than its tile) loads
    // cell nx + R - 1 in those unread slots, so that every index stays within
    // one period of the box, where the compare-and-add wrap holds (n >= 8 > R).
    auto wxy = [&](int xx, int yy) -> long long {
        if constexpr (wrap_table)
            return sWx[xx] + sWy[yy];
        else
            return wrap1(min(i0 - R + xx, nx + R - 1), nx) +
                   (long long)nx * wrap1(min(j0 - R + yy, ny + R - 1), ny);
    };
    auto issue = [&](int k, int buf) {
        const long long plane = sz * k;
        for (int t = tid; t < TY * (TX + 2 * R); t += TX * TY) {
            int yy = t / (TX + 2 * R), xx = t - yy * (TX + 2 * R);
            long long g = plane + wxy(xx, yy + R);
#pragma unroll
            for (int f = 0; f < 4; ++f) cp_async_elem(&sX[buf][f][yy][xx], vbase + cx[f] * np + g);
        }
        for (int t = tid; t < (TY + 2 * R) * TX; t += TX * TY) {
            int yy = t / TX, xx = t - yy * TX;
            long long g = plane + wxy(xx + R, yy);
#pragma unroll
            for (int f = 0; f < 4; ++f) cp_async_elem(&sY[buf][f][yy][xx], vbase + cy[f] * np + g);
        }
    };
    B qz[4][QD];
    if (VIS) {
        issue(k0, 0);
        cp_async_commit();
#pragma unroll
        for (int s = 0; s < 2 * R; ++s) {
            long long g = col + sz * pmod(k0 - R + s, nz);
#pragma unroll
            for (int f = 0; f < 4; ++f) qz[f][s] = active ? vbase[cz[f] * np + g] : B(0);
        }
    }
    double res = 0.0;
    bool bad = false;
    for (int k = k0; k < kend; ++k) {
        const int buf = (k - k0) & 1;
        const long long g = col + sz * k;
        if (VIS) {
            if (k + 1 < kend) issue(k + 1, buf ^ 1);
            cp_async_commit();
            long long g6 = col + sz * (k + R < nz ? k + R : k + R - nz);  // nz >= 8
#pragma unroll
            for (int f = 0; f < 4; ++f) qz[f][2 * R] = active ? vbase[cz[f] * np + g6] : B(0);
        }
        // pointwise operands, loaded before the wait so their latency overlaps
        B Rv[5];
        double ui[5], u_n[5];
        if (active) {
#pragma unroll
            for (int e = 0; e < 5; ++e) {
                Rv[e] = rbase[e * np + g];
                if (stage >= 0) ui[e] = uinb[e * np + g];
                if (stage >= 1) u_n[e] = unb[e * np + g];
            }
        }
        if (VIS) {
            cp_async_wait1();
            __syncthreads();
        }
        if (active) {
            if (VIS) {
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    const int c = tx + R, rr = ty + R;
                    const B *X = sX[buf][f][ty];
                    B dfx, dfy, dfz;
                    if constexpr (R == 3) {
                        dfx = cd6<B>(X[c - 3], X[c - 2], X[c - 1], X[c + 1], X[c + 2], X[c + 3],
                                     ixb);
                        dfy = cd6<B>(sY[buf][f][rr - 3][tx], sY[buf][f][rr - 2][tx],
                                     sY[buf][f][rr - 1][tx], sY[buf][f][rr + 1][tx],
                                     sY[buf][f][rr + 2][tx], sY[buf][f][rr + 3][tx], iyb);
                        dfz = cd6<B>(qz[f][0], qz[f][1], qz[f][2], qz[f][4], qz[f][5], qz[f][6],
                                     izb);
                    } else {
                        dfx = cd_any(X[c - 4], X[c - 3], X[c - 2], X[c - 1], X[c + 1], X[c + 2],
                                     X[c + 3], X[c + 4], bp.vcoef[0], ixb);
                        dfy = cd_any(sY[buf][f][rr - 4][tx], sY[buf][f][rr - 3][tx],
                                     sY[buf][f][rr - 2][tx], sY[buf][f][rr - 1][tx],
                                     sY[buf][f][rr + 1][tx], sY[buf][f][rr + 2][tx],
                                     sY[buf][f][rr + 3][tx], sY[buf][f][rr + 4][tx], bp.vcoef[1],
                                     iyb);
                        dfz = cd_any(qz[f][0], qz[f][1], qz[f][2], qz[f][3], qz[f][5], qz[f][6],
                                     qz[f][7], qz[f][8], bp.vcoef[2], izb);
                    }
                    B t = Rv[1 + f];
                    t -= dfx;
                    t -= dfy;
                    t -= dfz;
                    Rv[1 + f] = t;
                }
            }
            if (stage < 0) {
#pragma unroll
                for (int e = 0; e < 5; ++e) sa.rhs_out[5 * it.box + e][g] = double(Rv[e]);
            } else {
#pragma unroll
                for (int e = 0; e < 5; ++e) {
                    double rhs = -double(Rv[e]);
                    double out;
                    if (stage == 0) {
                        out = 1.0 * ui[e] + 1.0 * rhs * dt;
                    } else if (stage == 1) {
                        out = 0.75 * u_n[e] + 0.25 * (rhs * dt + ui[e]);
                    } else {
                        out = (1.0 / 3.0) * u_n[e] + (2.0 / 3.0) * (rhs * dt + ui[e]);
                        double dd = out - u_n[e];
                        res += dd * dd;
                    }
                    bad |= !isfinite(out);
                    uoutb[e * np + g] = out;
                }
            }
        }
        if (VIS) {
            __syncthreads();
#pragma unroll
            for (int s = 0; s < 2 * R; ++s)
#pragma unroll
                for (int f = 0; f < 4; ++f) qz[f][s] = qz[f][s + 1];
        }
    }
    if (bad) atomicOr(bd.flags, 1u);
    if (stage != 2) return;
    for (int o = 16; o > 0; o >>= 1) res += __shfl_xor_sync(0xffffffffu, res, o);
    if ((tid & 31) == 0) red[tid >> 5] = res;
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < TX * TY / 32; ++w) res += red[w];
        atomicAdd(bd.res_acc, res);
    }
}

namespace {
constexpr size_t visc_smem_bytes(int R) {
    // planes (row pitch TX + 8) and z refills, the offset table rounded up to
    // 16 bytes, two mbarriers, and the 128 bytes of alignment slack
    return sizeof(double) * 2 * 4 * ((TY + 2 * R) * (TX + 8) + TX * TY) +
           16 * ((TY + 2 * R) * (TX + 2 * R) * 4 / 16 + 1) + 2 * sizeof(unsigned long long) + 128;
}
// the R = 4 update kernel's x and y flux tiles (dynamic shared memory)
template <typename B>
constexpr size_t update_smem_bytes() {
    return sizeof(B) * 2 * 4 * (TY * (TX + 8) + (TY + 8) * TX);
}
template <typename B>
cudaError_t prepare_stencil_t() {
    cudaError_t e = cudaFuncSetAttribute(k_visc_flux25<B, 3>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)visc_smem_bytes(3));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_visc_flux25<B, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)visc_smem_bytes(4));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_update25<B, true, 4>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)update_smem_bytes<B>());
    return e;
}
}  // namespace

cudaError_t prepare_stencil_kernels(bool mixed) {
    return mixed ? prepare_stencil_t<float>() : prepare_stencil_t<double>();
}

template <typename B>
cudaError_t launch_visc_flux(const BoxDev *boxes, const WorkItem *items, int nitems, int kz,
                             int reach, cudaStream_t st) {
    if (nitems <= 0) return cudaSuccess;
    if (reach == 3)
        k_visc_flux25<B, 3><<<nitems, dim3(TX, TY), visc_smem_bytes(3), st>>>(boxes, items, kz);
    else
        k_visc_flux25<B, 4><<<nitems, dim3(TX, TY), visc_smem_bytes(4), st>>>(boxes, items, kz);
    return cudaGetLastError();
}

template <typename B>
cudaError_t launch_update(const BoxDev *boxes, const WorkItem *items, int nitems, int kz,
                          StageArgs sa, bool any_viscous, int reach, cudaStream_t st) {
    if (nitems <= 0) return cudaSuccess;
    if (!any_viscous)
        k_update25<B, false, 3><<<nitems, dim3(TX, TY), 0, st>>>(boxes, items, kz, sa);
    else if (reach == 3)
        k_update25<B, true, 3><<<nitems, dim3(TX, TY), 0, st>>>(boxes, items, kz, sa);
    else
        k_update25<B, true, 4><<<nitems, dim3(TX, TY), update_smem_bytes<B>(), st>>>(boxes, items,
                                                                                  kz, sa);
    return cudaGetLastError();
}

template cudaError_t launch_visc_flux<double>(const BoxDev *, const WorkItem *, int, int, int,
                                              cudaStream_t);
template cudaError_t launch_visc_flux<float>(const BoxDev *, const WorkItem *, int, int, int,
                                             cudaStream_t);
template cudaError_t launch_update<double>(const BoxDev *, const WorkItem *, int, int, StageArgs,
                                           bool, int, cudaStream_t);
template cudaError_t launch_update<float>(const BoxDev *, const WorkItem *, int, int, StageArgs,
                                          bool, int, cudaStream_t);

}  // namespace nuc3d
