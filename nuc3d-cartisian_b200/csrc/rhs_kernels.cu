// Batched whole-box kernels: primitive recovery, dt, residual and the
// directional WENO5 / WENO7 sweeps.
//
// One RK stage = k_inviscid<x> (which recovers the primitives of its tiles:
// k_prim's work; k_prim itself runs first for boxes whose x lines use the
// line kernel) -> [k_dt on the first stage] -> [k_visc_flux25] ->
// k_inviscid<y> -> k_inviscid<z> -> k_update25, each one launch for every
// box of a batch.
// The reference's per-direction rotated copies, halo buffers and MPI
// self-messages (euler3d.cpp:307-387, NaiverStokes3d.cpp:87-369,
// MPICommunicator.cpp:81-132) become periodic index wraps in the tile loads.
#include "nuc3d_device.cuh"
#include "prim_device.cuh"
#include "rhs_kernels.h"

namespace nuc3d {

// ----------------------------------------------------------------- k_prim --
// prim_cell, prim_store and eig_block_max: prim_device.cuh

// A work item is (box, first cell chunk, cell count).
__global__ void __launch_bounds__(256, 4) k_prim(const BoxDev *__restrict__ boxes,
                                                 const WorkItem *__restrict__ items, int in_slot,
                                                 int want_eig) {
    const WorkItem it = items[blockIdx.x];
    const BoxDev &bd = boxes[it.box];
    if (!bd.active) return;
    const long long np = bd.np;
    const double *__restrict__ q = fieldU(bd, in_slot, 0);
    const PrimConst pk(bd.p);
    double lx = 0.0, ly = 0.0, lz = 0.0;
    const long long n0 = (long long)it.a * kPrimChunk, n1 = n0 + it.b;
    // the next cell's state is loaded while the current one is converted
    long long n = n0 + threadIdx.x;
    double Qn[5];
#pragma unroll
    for (int e = 0; e < 5; ++e) Qn[e] = n < n1 ? q[e * np + n] : 1.0;
    for (; n < n1; n += blockDim.x) {
        double Q[5];
#pragma unroll
        for (int e = 0; e < 5; ++e) Q[e] = Qn[e];
        const long long nxt = n + blockDim.x;
        if (nxt < n1) {
#pragma unroll
            for (int e = 0; e < 5; ++e) Qn[e] = q[e * np + nxt];
        }
        PrimCell o;
        prim_cell(pk, Q, o);
        prim_store(bd, n, o);
        lx = fmax(add_(fabs(o.u), o.c), lx);
        ly = fmax(add_(fabs(o.v), o.c), ly);
        lz = fmax(add_(fabs(o.w), o.c), lz);
    }
    if (!want_eig) return;
    eig_block_max(bd, lx, ly, lz);
}

__global__ void k_clear_eig(const BoxDev *boxes, int nboxes) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nboxes || !boxes[b].active) return;
    boxes[b].eig[0] = boxes[b].eig[1] = boxes[b].eig[2] = 0.0;
}

// -------------------------------------------------------------------- k_dt --
// EulerData3D::getDt (euler3d.cpp:459-466) and PDEData3d::solve's
// dt_global = dt_local * cfl (PDEData3d.cpp:161-165).  One thread per box.
__global__ void k_dt(const BoxDev *boxes, int nboxes) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nboxes || !boxes[b].active) return;
    const BoxDev &bd = boxes[b];
    const double *eig = bd.eig;
    double dt_xi = bd.p.d[0] / eig[0];
    double dt_eta = bd.p.d[1] / eig[1];
    double dt_zeta = bd.p.d[2] / eig[2];
    double dt_local = 1.0 / (1.0 / dt_xi + 1.0 / dt_eta + 1.0 / dt_zeta);
    StepScalars *sc = bd.sc;
    sc->dt_local = dt_local;
    sc->dt = dt_local * sc->cfl;
    sc->dt_hist[sc->step % kHistory] = sc->dt;
}

// residual = sqrt(sum / (5 N)) / dt (PDEData3d.cpp:212); advances time and
// the step counter.  One thread per box.
__global__ void k_residual(const BoxDev *boxes, int nboxes) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nboxes || !boxes[b].active) return;
    const BoxDev &bd = boxes[b];
    StepScalars *sc = bd.sc;
    double r = sqrt(*bd.res_acc / (double)(bd.p.N * 5)) / sc->dt;
    sc->res_hist[sc->step % kHistory] = r;
    sc->time += sc->dt;
    sc->step += 1;
    *bd.res_acc = 0.0;
}

// -------------------------------------------------------------- k_inviscid --
// Tile of the directional sweep: TL lines x TC cells along the sweep; every
// thread owns one line and a run of R consecutive faces of it.  H is the
// stencil half-width (3 for WENO5, 4 for WENO7).  TCX is the tile length
// along the sweep, 32 or 64 cells (an autotuned shape: a 64-cell tile stages
// 64 + 2H cells instead of 32 + 2H, 8 % fewer split fluxes per cell for
// WENO5, at twice the shared memory per block).
//   DIR 0 (x): 16 lines (rows j) per tile; the runs of a line sit in
//              consecutive lanes of one warp (TCX / R <= 32).
//   DIR 1/2:   TL = one 128-byte row of B (16 FP64 / 32 FP32 columns i) per
//              tile; consecutive lanes are consecutive lines (coalesced).
template <int DIR, typename B, int RUN, int H = 3, int TCX = 32>
struct InvGeom {
    static_assert(TCX == 32 || TCX == 64, "tile length");
    static_assert(DIR != 0 || TCX / RUN <= 32, "the x sweep's runs of a line share a warp");
    static constexpr int R = RUN;               // faces per thread (1, 2 or 4)
    static constexpr int NR = TCX / RUN;        // runs per line
    static constexpr int TC = R * NR;           // cells per tile along the sweep (32 or 64)
    static constexpr int TL = DIR == 0 ? 16 : 128 / (int)sizeof(B);
    static constexpr int NF = TC + 2 * H;       // staged cells (H-cell halo each side)
    static constexpr int S = (NF + R - 1) / R;  // DIR 0 interleave stride
    static constexpr int NT = TL * NR;          // threads
    static constexpr int SF = DIR == 0 ? TL * R * S : NF * TL;  // staged values per flux
    static constexpr size_t SMEM = sizeof(B) * (size_t)(10 * SF + 2 * NT);  // dynamic
    // WENO5, 32-cell tiles: the staged tile (~52 KB) admits 4 blocks per SM;
    // blocks of up to 256 threads are held to the registers that keep all 4
    // resident, larger ones to 64 registers per thread.  The FP32 4-face x
    // tile (28 KB) is held to 6 blocks (80 registers; measured faster than 4
    // or 8).  64-cell tiles: as many blocks as their shared memory admits, at
    // most 4 and at most 1024 threads per SM in all (at least 64 registers
    // per thread).  (WENO7's sweep has its own kernel without a register
    // cap.)
    static constexpr int FIT = (int)((size_t)220 * 1024 / (SMEM + 1024));
    static constexpr int MINB64 = FIT < 1 ? 1 : (FIT > 4 ? 4 : FIT);
    static constexpr int CAP64 = 1024 / NT < 1 ? 1 : 1024 / NT;
    static constexpr int MINB =
        TCX == 64 ? (MINB64 < CAP64 ? MINB64 : CAP64)
                  : (NT <= 256 ? ((DIR == 0 && sizeof(B) == 4 && NT == 128) ? 6 : 4) : 1024 / NT);
    // thread -> (line, run)
    __device__ static void thread(int t, int &l, int &r) {
        if (DIR == 0) {
            l = t / NR;
            r = t % NR;
        } else {
            l = t % TL;
            r = t / TL;
        }
    }
    // staged position pc (cell c0 - H + pc) of line l for flux v.  DIR 0
    // interleaves positions so that the runs of a line (stride R) read
    // consecutive words.
    __device__ static int sf(int v, int l, int pc) {
        return DIR == 0 ? v * SF + (l * R + pc % R) * S + pc / R : v * SF + pc * TL + l;
    }
    // staging loop: item t -> (line, position) with consecutive t reading
    // consecutive addresses
    __device__ static void stage_item(int t, int &l, int &pc) {
        if (DIR == 0) {
            l = t / NF;
            pc = t - l * NF;
        } else {
            l = t % TL;
            pc = t / TL;
        }
    }
};

// Inviscid flux derivative along DIR for all 5 equations (euler3d.cpp:307-387
// + combineFluxLR :23-56 + setDerivatives*Inv :143-253), with the box's
// point-wise flux split (LF, AUSM or AUSMp; split_prepare) done while
// staging.
//   accumulate = 0: R = dF/dx ; 1: R += dG/dy (the RHS summation order of
//   NaiverStokes3d.cpp:396-446).
// Work item: (box, a, b, c) = DIR 0: (x chunk, j group, k); DIR 1: (i group,
// y chunk, k); DIR 2: (i group, j, z chunk).
// Each thread computes F^ = F^+ + F^- on its R faces with a register sliding
// window (the second differences of the smoothness indicators are carried
// from face to face), takes the first face of the next run from a neighbour
// through shared memory, and writes dF for its R cells.
// Mixed precision (B = float): the split fluxes are formed in FP64 and each
// line's value at the tile's first interior cell is subtracted before
// rounding to FP32.  WENO5 commutes with adding a constant and the constant
// cancels in the face difference, so this only removes rounding error.
template <int SCHEME, int DIR, typename B, int RUN, int TCX>
__device__ __forceinline__ void inviscid_body(const BoxDev *__restrict__ boxes,
                                              const WorkItem *__restrict__ items, int in_slot,
                                              int accumulate, int prim_mode) {
    constexpr int H = scheme_halo(SCHEME);
    using G = InvGeom<DIR, B, RUN, H, TCX>;
    constexpr int TL = G::TL, TC = G::TC, NF = G::NF, R = G::R, NR = G::NR, NT = G::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    B *sF = reinterpret_cast<B *>(smem_raw);  // [10][SF] split fluxes (+ e, then - e)
    B *xb = sF + 10 * G::SF;                  // [2][NT] first face of each run
    __shared__ double sRef[10][TL];

    const WorkItem it = items[blockIdx.x];
    const BoxDev &bd = boxes[it.box];
    if (!bd.active) return;
    const BoxParams &bp = bd.p;
    const double *const qbase = fieldU(bd, in_slot, 0);
    const double *const wbase = fieldW(bd, 0);
    B *const rbase = fieldR<B>(bd, 0);
    const long long np = bd.np;
    const int n = bp.n[DIR];
    int l0, c0, fixed;  // first line, first cell of the chunk, the third index
    if (DIR == 0) {
        c0 = it.a * TC;
        l0 = it.b * TL;
        fixed = it.c;
    } else if (DIR == 1) {
        l0 = it.a * TL;
        c0 = it.b * TC;
        fixed = it.c;
    } else {
        l0 = it.a * TL;
        fixed = it.b;
        c0 = it.c * TC;
    }
    const int nl = DIR == 0 ? bp.n[1] : bp.n[0];  // extent of the line index
    const long long sy = bp.stride[1], sz = bp.stride[2];
    auto gidx = [&](int l, int pos) -> long long {
        int a = l0 + l;
        if (DIR == 0) return pos + sy * a + sz * fixed;
        if (DIR == 1) return a + sy * pos + sz * fixed;
        return a + sy * fixed + sz * pos;
    };
    const int riemann = bp.riemann;
    // prim_mode (x sweep only): 0 reads u_n, p, c from W; 1 recovers the
    // primitives from the state (prim_cell) and writes W for the tile's own
    // cells; 2 also folds their eigenvalues into the box's maxima
    const bool own_prim = DIR == 0 && prim_mode != 0;
    const PrimConst pk(bp);
    double eg[3] = {0.0, 0.0, 0.0};
    // split fluxes of cell g; store: g is one of the tile's own cells
    auto split = [&](long long g, double Fp[5], double Fm[5], bool store) {
        double Q[5];
#pragma unroll
        for (int e = 0; e < 5; ++e) Q[e] = qbase[e * np + g];
        double un, p, c;
        if (own_prim) {
            PrimCell o;
            prim_cell(pk, Q, o);
            un = o.u;
            p = o.p;
            c = o.c;
            if (store) {
                prim_store(bd, g, o);
                eg[0] = fmax(add_(fabs(o.u), o.c), eg[0]);
                eg[1] = fmax(add_(fabs(o.v), o.c), eg[1]);
                eg[2] = fmax(add_(fabs(o.w), o.c), eg[2]);
            }
        } else {
            un = wbase[DIR * np + g];
            p = wbase[3 * np + g];
            c = wbase[4 * np + g];
        }
        if (riemann == RIEMANN_LF) {  // block-uniform
            // physicsModel.cpp:546-565, spelt out for all five equations:
            // F+- = F/2 +- (lambda/2) Q with the halves taken first (exact)
            const double hun = mul_(0.5, un), hlam = mul_(0.5, add_(fabs(un), c));
            double hf[5];
#pragma unroll
            for (int e = 0; e < 4; ++e) hf[e] = mul_(hun, Q[e]);
            hf[1 + DIR] = fma_(hun, Q[1 + DIR], mul_(0.5, p));
            hf[4] = mul_(hun, add_(Q[4], p));
#pragma unroll
            for (int e = 0; e < 5; ++e) {
                Fp[e] = fma_(hlam, Q[e], hf[e]);
                Fm[e] = fma_(-hlam, Q[e], hf[e]);
            }
        } else {
            SplitCell sc;
            split_prepare(riemann, un, p, c, sc);
#pragma unroll
            for (int e = 0; e < 5; ++e) split_eq<DIR>(riemann, sc, e, Q[e], Fp[e], Fm[e]);
        }
    };
    const bool mixed = sizeof(B) == sizeof(float);
    if (mixed) {  // per-line reference values (cell c0, always inside the box)
        if (threadIdx.x < TL) {
            int l = threadIdx.x;
            double Fp[5], Fm[5];
            if (l0 + l < nl) {
                split(gidx(l, c0), Fp, Fm, false);
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
    // phase 1: stage the split fluxes of cells c0-H .. c0+TC+H-1
    auto stage_store = [&](int l, int pc, const double Fp[5], const double Fm[5]) {
#pragma unroll
        for (int e = 0; e < 5; ++e) {
            if (mixed) {
                sF[G::sf(e, l, pc)] = B(sub_(Fp[e], sRef[e][l]));
                sF[G::sf(5 + e, l, pc)] = B(sub_(Fm[e], sRef[5 + e][l]));
            } else {
                sF[G::sf(e, l, pc)] = B(Fp[e]);
                sF[G::sf(5 + e, l, pc)] = B(Fm[e]);
            }
        }
    };
    // position of staged cell pc in the box: in [-H, n + NF), wrapped
    // without a division (n >= 8 > H)
    auto stage_pos = [&](int pc) {
        int pos = c0 - H + pc;
        if (pos < 0) pos += n;
        while (pos >= n) pos -= n;
        return pos;
    };
    for (int t = threadIdx.x; t < TL * NF; t += NT) {
        int l, pc;
        G::stage_item(t, l, pc);
        double Fp[5], Fm[5];
        if (l0 + l < nl) {
            // the tile's own cells: staged positions H .. H+TC-1 inside the box
            const bool own = pc >= H && pc < H + TC && c0 + pc - H < n;
            split(gidx(l, stage_pos(pc)), Fp, Fm, own);
        } else {
#pragma unroll
            for (int e = 0; e < 5; ++e) Fp[e] = Fm[e] = 0.0;
        }
        stage_store(l, pc, Fp, Fm);
    }
    __syncthreads();
    // phase 2: runs of faces.  Face m (local) lies between cells c0+m-1 and
    // c0+m; '+' reads staged positions m..m+4, '-' reads m+5..m+1.
    int l, r;
    G::thread(threadIdx.x, l, r);
    const int m0 = r * R;
    const bool last = r == NR - 1;       // also computes face TC (next tile's first)
    const bool line_ok = l0 + l < nl;
    const bool zq = SCHEME == SCHEME_Z && (bp.quirks & QK_WENOZ_BETA2);
    const B inv_d = B(bp.inv_d[DIR]);
    int nbr_l, nbr_r = r + 1;            // the thread owning the next run
    nbr_l = l;
    const int nbr = DIR == 0 ? nbr_l * NR + nbr_r : nbr_r * TL + nbr_l;
#pragma unroll 1
    for (int e = 0; e < 5; ++e) {
        // the RHS values this equation adds to (y, z), loaded before the faces
        // so that their latency hides behind the reconstruction
        B racc[R];
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int gc = c0 + m0 + k;
            racc[k] = (accumulate && line_ok && gc < n) ? rbase[gidx(l, gc) + e * np] : B(0);
        }
        B Fh[R + 1];
        if constexpr (SCHEME == SCHEME_W7 && sizeof(B) == 4 && DIR == 0) {
            // FP32 weno7js, x sweep: faces in pairs on the packed f32x2 arithmetic, '+'
            // in ascending order (positions m..m+6) beside '-' in descending
            // order (positions m'+7..m'+1), whose windows step alike (drop f0,
            // gain f6); component-wise the operations of weno7_face, so every
            // face is bitwise the one-sided form's (the WENO5 x sweep below
            // pairs its faces the same way).  256^3 mixed x sweeps 2.55 ->
            // 2.43 ms per step; in the y/z sweeps the joint window's registers
            // (up to 122) cost more than the packing saves (2.15 -> 2.22 and
            // 2.20 -> 2.31 ms), so they keep the one-sided windows.
            const int K = R + (last ? 1 : 0);
            const int mq = m0 + K - 1;  // the '-' side's first face
            float2 f[7];
#pragma unroll
            for (int j = 0; j < 7; ++j)
                f[j] = make_float2(sF[G::sf(e, l, m0 + j)], sF[G::sf(5 + e, l, mq + 7 - j)]);
            float gp[R + 1], gm[R + 1];
#pragma unroll
            for (int j = 0; j <= R; ++j) {
                if (j == R && !last) break;
                const float2 fr = weno7_face2(f[0], f[1], f[2], f[3], f[4], f[5], f[6]);
                gp[j] = fr.x;
                gm[j] = fr.y;
                if (j + 1 < K) {
#pragma unroll
                    for (int i = 0; i < 6; ++i) f[i] = f[i + 1];
                    // '+' gains position m0+j+7, '-' position m0+K-1-j
                    f[6] = make_float2(sF[G::sf(e, l, m0 + j + 7)], sF[G::sf(5 + e, l, mq - j)]);
                }
            }
#pragma unroll
            for (int k = 0; k <= R; ++k) {
                if (k == R && !last) break;
                const float fmk = last ? gm[R - k] : gm[k < R ? R - 1 - k : 0];
                Fh[k] = add_(gp[k], fmk);
            }
        } else if constexpr (SCHEME == SCHEME_W7 || SCHEME == SCHEME_H78) {
            // face m: '+' reads positions m..m+6 (cells m-4..m+2), '-' reads
            // m+7..m+1 (cells m+3..m-3).  hccs78 blends faces 4..n-4 with the
            // central value of cells m-4..m+3 (positions m..m+7): its '+'
            // window carries position m+7 in f[7], its '-' window position m.
            constexpr bool h78 = SCHEME == SCHEME_H78;
            auto blended = [&](int k) {
                const int gm = c0 + m0 + k;
                return h78 && gm >= 4 && gm <= n - 4;
            };
            B f[8];
#pragma unroll
            for (int j = 0; j < 7; ++j) f[j] = sF[G::sf(e, l, m0 + j)];
            if (h78) f[7] = sF[G::sf(e, l, m0 + 7)];
#pragma unroll
            for (int k = 0; k <= R; ++k) {
                if (k == R && !last) break;
                if (blended(k))
                    Fh[k] = hccs78_face(f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[0], f[1], f[2],
                                        f[3], f[4], f[5], f[6], f[7]);
                else
                    Fh[k] = weno7_face(f[0], f[1], f[2], f[3], f[4], f[5], f[6]);
                if (k < R) {
#pragma unroll
                    for (int j = 0; j < 6; ++j) f[j] = f[j + 1];
                    if (h78) {
                        f[6] = f[7];
                        f[7] = sF[G::sf(e, l, m0 + k + 8)];
                    } else {
                        f[6] = sF[G::sf(e, l, m0 + k + 7)];
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 7; ++j) f[j] = sF[G::sf(5 + e, l, m0 + 7 - j)];
            if (h78) f[7] = sF[G::sf(5 + e, l, m0)];
#pragma unroll
            for (int k = 0; k <= R; ++k) {
                if (k == R && !last) break;
                if (blended(k))
                    Fh[k] = add_(Fh[k], hccs78_face(f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7],
                                                    f[6], f[5], f[4], f[3], f[2], f[1], f[0]));
                else
                    Fh[k] = add_(Fh[k], weno7_face(f[0], f[1], f[2], f[3], f[4], f[5], f[6]));
                if (k < R) {
                    if (h78) f[7] = f[6];  // position m+1 of the next face
#pragma unroll
                    for (int j = 6; j > 0; --j) f[j] = f[j - 1];
                    f[0] = (m0 + k + 8 < NF) ? sF[G::sf(5 + e, l, m0 + k + 8)] : B(0);
                }
            }
        } else if constexpr (SCHEME == SCHEME_W3 || SCHEME == SCHEME_U1) {
            // weno3js: face m from positions m..m+2 ('+', cells m-2..m) and
            // m+3..m+1 ('-'); upwind1st: position m ('+', cell m-1) and m+1
            // ('-', cell m)
#pragma unroll
            for (int k = 0; k <= R; ++k) {
                if (k == R && !last) break;
                const int m = m0 + k;
                if (SCHEME == SCHEME_U1)
                    Fh[k] = add_(sF[G::sf(e, l, m)], sF[G::sf(5 + e, l, m + 1)]);
                else
                    Fh[k] = add_(weno3js_face(sF[G::sf(e, l, m)], sF[G::sf(e, l, m + 1)],
                                              sF[G::sf(e, l, m + 2)]),
                                 weno3js_face(sF[G::sf(5 + e, l, m + 3)],
                                              sF[G::sf(5 + e, l, m + 2)],
                                              sF[G::sf(5 + e, l, m + 1)]));
            }
        } else {
            // FP64 runs of 4 faces step both windows together; the others step
            // them one after the other (measured faster for FP32, and the joint
            // form does not fit the 64-register budget of FP64 runs of 1 or 2)
            constexpr bool joint = sizeof(B) == 8 && R == 4;
            if constexpr (joint) {
                // WENO5: each window carries the first differences a_ij, the second
                // differences D and dd = 4 (13/12) D^2 of its current stencil, so each
                // new face adds one value, one difference, one second difference
                // and one square (weno5_face_dq).  The '+' stencil of face m is
                // positions m..m+4, the '-' stencil m+5..m+1; both windows step
                // together so that each face offers two independent chains.
                const int vp = e, vm = 5 + e;
                B p2 = sF[G::sf(vp, l, m0 + 2)], p3 = sF[G::sf(vp, l, m0 + 3)];
                B p4 = sF[G::sf(vp, l, m0 + 4)];
                B pa21, pa32, pa43, pD0, pD1, pD2;
                {
                    const B p0 = sF[G::sf(vp, l, m0)], p1 = sF[G::sf(vp, l, m0 + 1)];
                    const B pa10 = sub_(p1, p0);
                    pa21 = sub_(p2, p1);
                    pa32 = sub_(p3, p2);
                    pa43 = sub_(p4, p3);
                    pD0 = sub_(pa21, pa10);
                    pD1 = sub_(pa32, pa21);
                    pD2 = sub_(pa43, pa32);
                }
                B pdd0 = dd_of(pD0), pdd1 = dd_of(pD1), pdd2 = dd_of(pD2);
                B q0 = sF[G::sf(vm, l, m0 + 5)], q1 = sF[G::sf(vm, l, m0 + 4)];
                B q2 = sF[G::sf(vm, l, m0 + 3)];
                B qa10, qa21, qa32, qa43, qD0, qD1, qD2;
                {
                    const B q3 = sF[G::sf(vm, l, m0 + 2)], q4 = sF[G::sf(vm, l, m0 + 1)];
                    qa10 = sub_(q1, q0);
                    qa21 = sub_(q2, q1);
                    qa32 = sub_(q3, q2);
                    qa43 = sub_(q4, q3);
                    qD0 = sub_(qa21, qa10);
                    qD1 = sub_(qa32, qa21);
                    qD2 = sub_(qa43, qa32);
                }
                B qdd0 = dd_of(qD0), qdd1 = dd_of(qD1), qdd2 = dd_of(qD2);
                auto face = [&](int k) {
                    const int gm = c0 + m0 + k;
                    // weno5z.cpp:80 on the inner '+' faces 3..n-3: beta2's first
                    // term reads f2 - 2 f3 + f3 = -a32
                    const B dd2s = (zq && gm >= 3 && gm <= n - 3) ? dd_of(pa32) : pdd2;
                    const B fp = weno5_face_dq<SCHEME, B>(p2, pa21, pa32, pa43, pD0, pD2, pdd0, pdd1, dd2s);
                    const B fm = weno5_face_dq<SCHEME, B>(q2, qa21, qa32, qa43, qD0, qD2, qdd0, qdd1, qdd2);
                    return add_(fp, fm);
                };
    #pragma unroll
                for (int k = 0; k < R; ++k) {
                    Fh[k] = face(k);
                    // '+' gains position m0+k+5, '-' gains position m0+k+6
                    p2 = p3;
                    p3 = p4;
                    p4 = sF[G::sf(vp, l, m0 + k + 5)];
                    pa21 = pa32;
                    pa32 = pa43;
                    pa43 = sub_(p4, p3);
                    pD0 = pD1;
                    pD1 = pD2;
                    pD2 = sub_(pa43, pa32);
                    pdd0 = pdd1;
                    pdd1 = pdd2;
                    pdd2 = dd_of(pD2);
                    const B qn = (m0 + k + 6 < NF) ? sF[G::sf(vm, l, m0 + k + 6)] : B(0);
                    q2 = q1;
                    q1 = q0;
                    q0 = qn;
                    qa43 = qa32;
                    qa32 = qa21;
                    qa21 = qa10;
                    qa10 = sub_(q1, q0);
                    qD2 = qD1;
                    qD1 = qD0;
                    qD0 = sub_(qa21, qa10);
                    qdd2 = qdd1;
                    qdd1 = qdd0;
                    qdd0 = dd_of(qD0);
                }
                if (last) Fh[R] = face(R);
            } else if constexpr (sizeof(B) == 4 && DIR == 0) {
                // FP32 x sweep: faces in pairs on the packed f32x2 arithmetic.  The
                // thread's K faces (R, and the next run's first on the last
                // run) are taken '+' in ascending order beside '-' in
                // descending order: the '+' stencil of face m0+j (positions
                // m..m+4) and the '-' stencil of face m0+K-1-j (positions
                // m'+5..m'+1) both step by dropping f0 and gaining a new f4,
                // so one packed window (component x: '+', y: '-') carries
                // both.  Component-wise the operations are those of the
                // one-sided windows below, so every face is bitwise the same.
                // (256^3 mixed step, x sweeps: WENO5-Z 1.895 -> 1.84 ms, WENO5-JS
                // 1.81 -> 1.75 ms.  The y/z sweeps wait on their staging loads,
                // not on FP32 issue: there the packed form measured the same
                // (WENO5-Z) or 2-4 % slower (WENO5-JS), so they keep the
                // one-sided form.)
                const int K = R + (last ? 1 : 0);
                const int mq = m0 + K - 1;  // the '-' side's first face
                const int vp = e, vm = 5 + e;
                float2 w0 = make_float2(sF[G::sf(vp, l, m0)], sF[G::sf(vm, l, mq + 5)]);
                float2 w1 = make_float2(sF[G::sf(vp, l, m0 + 1)], sF[G::sf(vm, l, mq + 4)]);
                float2 X2 = make_float2(sF[G::sf(vp, l, m0 + 2)], sF[G::sf(vm, l, mq + 3)]);
                float2 X3 = make_float2(sF[G::sf(vp, l, m0 + 3)], sF[G::sf(vm, l, mq + 2)]);
                float2 X4 = make_float2(sF[G::sf(vp, l, m0 + 4)], sF[G::sf(vm, l, mq + 1)]);
                const float2 A10 = sub2_(w1, w0);
                float2 A21 = sub2_(X2, w1), A32 = sub2_(X3, X2), A43 = sub2_(X4, X3);
                float2 D0 = sub2_(A21, A10), D1 = sub2_(A32, A21), D2 = sub2_(A43, A32);
                float2 DD0 = dd2_of(D0), DD1 = dd2_of(D1), DD2 = dd2_of(D2);
                float gp[R + 1], gm[R + 1];
    #pragma unroll
                for (int j = 0; j <= R; ++j) {
                    if (j == R && !last) break;
                    const int gmp = c0 + m0 + j;
                    // weno5z.cpp:80 on the inner '+' faces 3..n-3 (x only)
                    float2 DD2s = DD2;
                    if (zq && gmp >= 3 && gmp <= n - 3) DD2s.x = dd_of(A32.x);
                    const float2 fr =
                        weno5_face_dq2<SCHEME>(X2, A21, A32, A43, D0, D2, DD0, DD1, DD2s);
                    gp[j] = fr.x;
                    gm[j] = fr.y;
                    if (j + 1 < K) {
                        // '+' gains position m0+j+5, '-' position m0+K-1-j
                        const float2 nw =
                            make_float2(sF[G::sf(vp, l, m0 + j + 5)], sF[G::sf(vm, l, mq - j)]);
                        X2 = X3;
                        X3 = X4;
                        X4 = nw;
                        A21 = A32;
                        A32 = A43;
                        A43 = sub2_(X4, X3);
                        D0 = D1;
                        D1 = D2;
                        D2 = sub2_(A43, A32);
                        DD0 = DD1;
                        DD1 = DD2;
                        DD2 = dd2_of(D2);
                    }
                }
                // face k: '+' value gp[k], '-' value gm[K-1-k]
    #pragma unroll
                for (int k = 0; k <= R; ++k) {
                    if (k == R && !last) break;
                    const float fmk = last ? gm[R - k] : gm[k < R ? R - 1 - k : 0];
                    Fh[k] = add_(gp[k], fmk);
                }
            } else {
                // WENO5: the window carries the first differences a_ij, the second
                // differences D and dd = 4 (13/12) D^2 of the current stencil, so each
                // new face adds one value, one difference, one second difference
                // and one square (weno5_face_dq).
                {  // '+' side: stencil f0..f4 = positions m..m+4
                    const int v = e;
                    B f0 = sF[G::sf(v, l, m0)], f1 = sF[G::sf(v, l, m0 + 1)];
                    B f2 = sF[G::sf(v, l, m0 + 2)], f3 = sF[G::sf(v, l, m0 + 3)];
                    B f4 = sF[G::sf(v, l, m0 + 4)];
                    B a10 = sub_(f1, f0), a21 = sub_(f2, f1), a32 = sub_(f3, f2), a43 = sub_(f4, f3);
                    B D0 = sub_(a21, a10), D1 = sub_(a32, a21), D2 = sub_(a43, a32);
                    B dd0 = dd_of(D0), dd1 = dd_of(D1), dd2 = dd_of(D2);
    #pragma unroll
                    for (int k = 0; k <= R; ++k) {
                        if (k == R && !last) break;
                        const int gm = c0 + m0 + k;
                        // weno5z.cpp:80 on the inner '+' faces 3..n-3: beta2's first
                        // term reads f2 - 2 f3 + f3 = -a32
                        const B dd2s = (zq && gm >= 3 && gm <= n - 3) ? dd_of(a32) : dd2;
                        Fh[k] = weno5_face_dq<SCHEME, B>(f2, a21, a32, a43, D0, D2, dd0, dd1, dd2s);
                        if (k < R) {
                            f2 = f3;
                            f3 = f4;
                            f4 = sF[G::sf(v, l, m0 + k + 5)];
                            a21 = a32;
                            a32 = a43;
                            a43 = sub_(f4, f3);
                            D0 = D1;
                            D1 = D2;
                            D2 = sub_(a43, a32);
                            dd0 = dd1;
                            dd1 = dd2;
                            dd2 = dd_of(D2);
                        }
                    }
                }
                {  // '-' side: stencil f0..f4 = positions m+5..m+1
                    const int v = 5 + e;
                    B f0 = sF[G::sf(v, l, m0 + 5)], f1 = sF[G::sf(v, l, m0 + 4)];
                    B f2 = sF[G::sf(v, l, m0 + 3)], f3 = sF[G::sf(v, l, m0 + 2)];
                    B f4 = sF[G::sf(v, l, m0 + 1)];
                    B a10 = sub_(f1, f0), a21 = sub_(f2, f1), a32 = sub_(f3, f2), a43 = sub_(f4, f3);
                    B D0 = sub_(a21, a10), D1 = sub_(a32, a21), D2 = sub_(a43, a32);
                    B dd0 = dd_of(D0), dd1 = dd_of(D1), dd2 = dd_of(D2);
    #pragma unroll
                    for (int k = 0; k <= R; ++k) {
                        if (k == R && !last) break;
                        Fh[k] = add_(Fh[k], weno5_face_dq<SCHEME, B>(f2, a21, a32, a43, D0, D2, dd0,
                                                                     dd1, dd2));
                        if (k < R) {
                            const B fn = (m0 + k + 6 < NF) ? sF[G::sf(v, l, m0 + k + 6)] : B(0);
                            f2 = f1;
                            f1 = f0;
                            f0 = fn;
                            a43 = a32;
                            a32 = a21;
                            a21 = a10;
                            a10 = sub_(f1, f0);
                            D2 = D1;
                            D1 = D0;
                            D0 = sub_(a21, a10);
                            dd2 = dd1;
                            dd1 = dd0;
                            dd0 = dd_of(D0);
                        }
                    }
                }
            }
        }
        // the first face of the next run: in the x sweep the runs of a line
        // are consecutive lanes of one warp (a shuffle, no barrier); in y/z
        // the next run may sit in another warp (shared memory)
        B next;
        if constexpr (DIR == 0) {
            const B nb = __shfl_down_sync(0xffffffffu, Fh[0], 1);
            next = last ? Fh[R] : nb;
        } else {
            B *x = xb + (e & 1) * NT;
            x[threadIdx.x] = Fh[0];
            __syncthreads();
            next = last ? Fh[R] : x[nbr];
        }
        if (line_ok) {
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int gc = c0 + m0 + k;
                if (gc >= n) break;
                B hi = (k + 1 < R) ? Fh[k + 1] : next;
                B dfe = mul_(sub_(hi, Fh[k]), inv_d);
                rbase[gidx(l, gc) + e * np] = accumulate ? add_(racc[k], dfe) : dfe;
            }
        }
    }
    if (own_prim && prim_mode == 2) eig_block_max(bd, eg[0], eg[1], eg[2]);
}

// The WENO5 sweeps carry a register cap (InvGeom::MINB); the WENO7 sweep is
// compiled without one (its own kernel, so that the register allocation is
// left to the compiler's default).
template <int SCHEME, int DIR, typename B, int RUN, int TCX>
__global__ void __launch_bounds__(InvGeom<DIR, B, RUN, 3, TCX>::NT, InvGeom<DIR, B, RUN, 3, TCX>::MINB)
    k_inviscid(const BoxDev *__restrict__ boxes, const WorkItem *__restrict__ items, int in_slot,
               int accumulate, int prim_mode) {
    inviscid_body<SCHEME, DIR, B, RUN, TCX>(boxes, items, in_slot, accumulate, prim_mode);
}
// WENO7 and hccs78 (4-cell halos)
template <int SCHEME, int DIR, typename B, int RUN, int TCX>
__global__ void __launch_bounds__(InvGeom<DIR, B, RUN, 4, TCX>::NT)
    k_inviscid_w7(const BoxDev *__restrict__ boxes, const WorkItem *__restrict__ items,
                  int in_slot, int accumulate, int prim_mode) {
    inviscid_body<SCHEME, DIR, B, RUN, TCX>(boxes, items, in_slot, accumulate, prim_mode);
}

using InvKernel = void (*)(const BoxDev *, const WorkItem *, int, int, int);
template <int SCHEME, int DIR, typename B, int RUN, int TCX>
static InvKernel inv_kernel() {
    if constexpr (SCHEME == SCHEME_W7 || SCHEME == SCHEME_H78)
        return k_inviscid_w7<SCHEME, DIR, B, RUN, TCX>;
    else
        return k_inviscid<SCHEME, DIR, B, RUN, TCX>;
}

// --------------------------------------------------------------- launches --
template <int SCHEME, int DIR, typename B, int RUN, int TCX>
static size_t inv_smem_t() {
    return InvGeom<DIR, B, RUN, scheme_halo(SCHEME), TCX>::SMEM;
}

InvTileDims inviscid_tile(int dir, bool mixed, int tile_cells) {
    // the lines per tile are the same for every run length and tile length
    const int tl = dir == 0 ? InvGeom<0, double, 1>::TL
                            : (mixed ? InvGeom<1, float, 1>::TL : InvGeom<1, double, 1>::TL);
    return InvTileDims{tl, tile_cells};
}

template <int SCHEME, int DIR, typename B, int RUN, int TCX>
static cudaError_t launch_t(const BoxDev *boxes, const WorkItem *items, int nitems, int in_slot,
                            int accumulate, int prim_mode, cudaStream_t st) {
    using G = InvGeom<DIR, B, RUN, scheme_halo(SCHEME), TCX>;
    if (nitems <= 0) return cudaSuccess;
    inv_kernel<SCHEME, DIR, B, RUN, TCX>()<<<nitems, G::NT, inv_smem_t<SCHEME, DIR, B, RUN, TCX>(),
                                             st>>>(boxes, items, in_slot, accumulate, prim_mode);
    return cudaGetLastError();
}

// variant v: kInvTileCells[v] cells per tile, kInvRunLen[v] faces per thread
template <int SCHEME, int DIR, typename B>
static cudaError_t launch_v(int variant, const BoxDev *boxes, const WorkItem *items, int nitems,
                            int in_slot, int accumulate, int prim_mode, cudaStream_t st) {
    switch (variant) {
        case 0: return launch_t<SCHEME, DIR, B, 1, 32>(boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        case 1: return launch_t<SCHEME, DIR, B, 2, 32>(boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        case 3: return launch_t<SCHEME, DIR, B, 2, 64>(boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        case 4: return launch_t<SCHEME, DIR, B, 4, 64>(boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        default: return launch_t<SCHEME, DIR, B, 4, 32>(boxes, items, nitems, in_slot, accumulate, prim_mode, st);
    }
}

template <typename B>
cudaError_t launch_inviscid(int scheme, int dir, int variant, const BoxDev *boxes,
                            const WorkItem *items, int nitems, int in_slot, int accumulate,
                            int prim_mode, cudaStream_t st) {
    if (nitems <= 0) return cudaSuccess;
    if (scheme == SCHEME_JS) {
        if (dir == 0) return launch_v<SCHEME_JS, 0, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        if (dir == 1) return launch_v<SCHEME_JS, 1, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        return launch_v<SCHEME_JS, 2, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
    }
    if (scheme == SCHEME_Z) {
        if (dir == 0) return launch_v<SCHEME_Z, 0, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        if (dir == 1) return launch_v<SCHEME_Z, 1, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        return launch_v<SCHEME_Z, 2, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
    }
    if (scheme == SCHEME_W7) {
        if (dir == 0) return launch_v<SCHEME_W7, 0, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        if (dir == 1) return launch_v<SCHEME_W7, 1, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        return launch_v<SCHEME_W7, 2, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
    }
    if (scheme == SCHEME_H78) {
        if (dir == 0) return launch_v<SCHEME_H78, 0, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        if (dir == 1) return launch_v<SCHEME_H78, 1, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        return launch_v<SCHEME_H78, 2, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
    }
    if (scheme == SCHEME_W3) {
        if (dir == 0) return launch_v<SCHEME_W3, 0, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        if (dir == 1) return launch_v<SCHEME_W3, 1, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        return launch_v<SCHEME_W3, 2, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
    }
    if (scheme == SCHEME_U1) {
        if (dir == 0) return launch_v<SCHEME_U1, 0, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        if (dir == 1) return launch_v<SCHEME_U1, 1, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
        return launch_v<SCHEME_U1, 2, B>(variant, boxes, items, nitems, in_slot, accumulate, prim_mode, st);
    }
    return cudaErrorInvalidValue;
}

template <int SCHEME, int DIR, typename B, int RUN, int TCX>
static cudaError_t prepare_t() {
    return cudaFuncSetAttribute(inv_kernel<SCHEME, DIR, B, RUN, TCX>(),
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)inv_smem_t<SCHEME, DIR, B, RUN, TCX>());
}
template <int SCHEME, int DIR, typename B>
static cudaError_t prepare_runs() {
    cudaError_t e[kInvVariants] = {prepare_t<SCHEME, DIR, B, 1, 32>(), prepare_t<SCHEME, DIR, B, 2, 32>(),
                                   prepare_t<SCHEME, DIR, B, 4, 32>(), prepare_t<SCHEME, DIR, B, 2, 64>(),
                                   prepare_t<SCHEME, DIR, B, 4, 64>()};
    for (cudaError_t x : e)
        if (x != cudaSuccess) return x;
    return cudaSuccess;
}
template <typename B>
static cudaError_t prepare_all() {
    cudaError_t e[18] = {prepare_runs<SCHEME_JS, 0, B>(), prepare_runs<SCHEME_JS, 1, B>(),
                         prepare_runs<SCHEME_JS, 2, B>(), prepare_runs<SCHEME_Z, 0, B>(),
                         prepare_runs<SCHEME_Z, 1, B>(), prepare_runs<SCHEME_Z, 2, B>(),
                         prepare_runs<SCHEME_W7, 0, B>(), prepare_runs<SCHEME_W7, 1, B>(),
                         prepare_runs<SCHEME_W7, 2, B>(), prepare_runs<SCHEME_H78, 0, B>(),
                         prepare_runs<SCHEME_H78, 1, B>(), prepare_runs<SCHEME_H78, 2, B>(),
                         prepare_runs<SCHEME_W3, 0, B>(), prepare_runs<SCHEME_W3, 1, B>(),
                         prepare_runs<SCHEME_W3, 2, B>(), prepare_runs<SCHEME_U1, 0, B>(),
                         prepare_runs<SCHEME_U1, 1, B>(), prepare_runs<SCHEME_U1, 2, B>()};
    for (cudaError_t x : e)
        if (x != cudaSuccess) return x;
    return cudaSuccess;
}

cudaError_t prepare_inviscid_kernels(bool mixed) {
    return mixed ? prepare_all<float>() : prepare_all<double>();
}

cudaError_t launch_prim(const BoxDev *boxes, const WorkItem *items, int nitems, int in_slot,
                        int want_eig, cudaStream_t st) {
    if (nitems <= 0) return cudaSuccess;
    k_prim<<<nitems, 256, 0, st>>>(boxes, items, in_slot, want_eig);
    return cudaGetLastError();
}

cudaError_t launch_clear_eig(const BoxDev *boxes, int nboxes, cudaStream_t st) {
    k_clear_eig<<<(nboxes + 127) / 128, 128, 0, st>>>(boxes, nboxes);
    return cudaGetLastError();
}

cudaError_t launch_dt(const BoxDev *boxes, int nboxes, cudaStream_t st) {
    k_dt<<<(nboxes + 127) / 128, 128, 0, st>>>(boxes, nboxes);
    return cudaGetLastError();
}

cudaError_t launch_residual(const BoxDev *boxes, int nboxes, cudaStream_t st) {
    k_residual<<<(nboxes + 127) / 128, 128, 0, st>>>(boxes, nboxes);
    return cudaGetLastError();
}

template cudaError_t launch_inviscid<double>(int, int, int, const BoxDev *, const WorkItem *, int,
                                             int, int, int, cudaStream_t);
template cudaError_t launch_inviscid<float>(int, int, int, const BoxDev *, const WorkItem *, int,
                                            int, int, int, cudaStream_t);
}  // namespace nuc3d
