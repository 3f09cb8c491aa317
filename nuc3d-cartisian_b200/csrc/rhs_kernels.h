// Launch interface of the whole-box kernels.  Internal to the library; the
// public surface is the C ABI in include/nuc3d_b200.h.
//
// Every kernel is batched: it receives a device table of boxes (BoxDev: the
// box's parameters and field pointers) and a list of work items, one per
// thread block, each naming a box and a tile of it.  A batch of boxes of
// different sizes therefore advances with one launch per kernel class, and a
// single box is simply a batch of one.
#pragma once

#include <cuda_runtime.h>

#include "nuc3d_device.cuh"

namespace nuc3d {

constexpr int kHistory = 1024;  // per-box step history kept on the device

// Per-box scalars in device memory, so a step never waits on the host:
// dt of the current step, simulated time, the step counter that indexes the
// history (it lets a captured CUDA graph replay without new arguments).
struct StepScalars {
    double dt;
    double dt_local;
    double time;
    double cfl;
    long long step;
    long long pad;
    double dt_hist[kHistory];
    double res_hist[kHistory];
};

// One box of a batch as the kernels see it.  U[s]: conserved state of RK
// stage s (U[0] = u_n, updated in place by the last stage); W: u, v, w, p,
// c, T (FP64); R: inviscid RHS accumulator and V: viscous fluxes
// (tau_xx, tau_xy, tau_xz, tau_yy, tau_yz, tau_zz, E_x, E_y, E_z) in the bulk
// type.
struct BoxDev {
    BoxParams p;
    // All fields of the box live in one allocation at fixed offsets, so a
    // kernel needs only this base and the padded field length np:
    //   U[s][e] (stage s, equation e)  at base + (5 s + e) np   (FP64)
    //   W[i]                            at base + (15 + i) np   (FP64)
    //   R[e], V[i]  (bulk type B)       at (B *)(base + 21 np) + e np, + (5 + i) np
    double *base;
    long long np;
    double *eig;      // [3] running max eigenvalues of the current step
    double *res_acc;  // residual partial sum
    unsigned *flags;  // bit 0: non-finite state seen; bit 1: a bounded device wait timed out
    StepScalars *sc;
    int active;       // 0: the box is skipped by every kernel
    int pad;
    // TMA tensor maps (CUtensorMap, 128 B each, in the box's allocation) of
    // the primitives u, v, w, T: [0..3] halo-plane boxes, [4..7] tile boxes
    // (kViscTmaBox*); null when the box's rows are not TMA-aligned (odd nx)
    // or the box is inviscid
    const void *tmw;
};

constexpr unsigned kFlagNonFinite = 1u, kFlagWaitTimeout = 2u;
// boxes of the viscous-flux kernel's TMA loads (elements x, y, z): the
// tile's plane with a 3-cell halo, x widened to start on a 32-byte boundary,
// and the tile's own columns
constexpr int kViscTmaHaloX = 40, kViscTmaHaloY = 14, kViscTmaTileX = 32, kViscTmaTileY = 8;

__host__ __device__ __forceinline__ double *fieldU(const BoxDev &b, int s, int e) {
    return b.base + (long long)(5 * s + e) * b.np;
}
__host__ __device__ __forceinline__ double *fieldW(const BoxDev &b, int i) {
    return b.base + (long long)(15 + i) * b.np;
}
template <typename B>
__host__ __device__ __forceinline__ B *fieldR(const BoxDev &b, int e) {
    return reinterpret_cast<B *>(b.base + 21 * b.np) + (long long)e * b.np;
}
template <typename B>
__host__ __device__ __forceinline__ B *fieldV(const BoxDev &b, int i) {
    return reinterpret_cast<B *>(b.base + 21 * b.np) + (long long)(5 + i) * b.np;
}

// A work item: box index and up to three tile coordinates.
struct WorkItem {
    int box, a, b, c;
};

// Stage addressing: which U buffers are input/output of RK stage `stage`;
// stage -1 evaluates the RHS of U[0] and writes it to `rhs_out`.
struct StageArgs {
    int stage;
    int in_slot;             // U index read by the RHS (0, 1, 2)
    int out_slot;            // U index written by the update (1, 2, 0)
    double *const *rhs_out;  // device array of 5 pointers per box (stage -1 only)
};

// Tile geometry of the batched kernels (host and device agree on these).
struct InvTileDims {
    int TL, TC;  // lines per tile, cells per tile along the sweep
};
InvTileDims inviscid_tile(int dir, bool mixed, int tile_cells);
constexpr int kT25X = 32, kT25Y = 8;  // 2.5-D tile of the stencil kernels (x, y)
// pencil depths (planes per work item) the autotuner chooses from; the first
// is the default
constexpr int kPencilDepths[3] = {32, 16, 64};
constexpr int kPrimChunk = 4096;                  // cells per k_prim work item

// Opt the inviscid kernels of one precision into their dynamic shared
// memory size (once per device, before any launch or stream capture).
cudaError_t prepare_inviscid_kernels(bool mixed);
cudaError_t launch_prim(const BoxDev *boxes, const WorkItem *items, int nitems, int in_slot,
                        int want_eig, cudaStream_t st);
cudaError_t launch_dt(const BoxDev *boxes, int nboxes, cudaStream_t st);
cudaError_t launch_residual(const BoxDev *boxes, int nboxes, cudaStream_t st);
cudaError_t launch_clear_eig(const BoxDev *boxes, int nboxes, cudaStream_t st);
// variant v of the sweep kernel: tiles of kInvTileCells[v] cells along the
// sweep, runs of kInvRunLen[v] faces per thread (picked per scheme and
// direction by the engine's autotuner); variants 0-2 use 32-cell tiles, 3-4
// 64-cell tiles (their work items differ: kInvTileClass)
constexpr int kInvVariants = 5;
constexpr int kInvTileCells[kInvVariants] = {32, 32, 32, 64, 64};
constexpr int kInvRunLen[kInvVariants] = {1, 2, 4, 2, 4};
constexpr int kInvTileClasses = 2;  // 32- and 64-cell tiles
constexpr int inv_tile_class(int variant) { return variant >= 3 ? 1 : 0; }
// scheme slots of the per-scheme sweep tables (indexed by scheme id; the
// line-solve schemes' slots (CRWENO5, hccs, hccs77) stay empty, their lines
// run in launch_crweno)
constexpr int kSchemes = 9;
// the line-solve schemes, in the order of the engine's line tables
constexpr int kLineSchemes = 3;
constexpr int kLineScheme[kLineSchemes] = {SCHEME_CR, SCHEME_HC, SCHEME_H77};
constexpr int line_slot(int scheme) {
    return scheme == SCHEME_CR ? 0 : (scheme == SCHEME_HC ? 1 : (scheme == SCHEME_H77 ? 2 : -1));
}
// prim_mode (x sweep only): 0 reads the primitives W; 1 recovers them from
// the state while staging and writes W for the tile's own cells (k_prim's
// work, bitwise the same); 2 also folds their eigenvalues into the boxes'
// running maxima (k_prim with want_eig)
template <typename B>
cudaError_t launch_inviscid(int scheme, int dir, int variant, const BoxDev *boxes,
                            const WorkItem *items, int nitems, int in_slot, int accumulate,
                            int prim_mode, cudaStream_t st);
// raises the dynamic shared-memory limits of the 2.5-D stencil kernels
cudaError_t prepare_stencil_kernels(bool mixed);
// Stencil classes of the 2.5-D kernels: boxes whose three directions use cd6
// (class 0, reach 3) and all others (class 1, reach 4: each direction's
// scheme as coefficients, BoxParams::vcoef).
constexpr int kVisClasses = 2;
constexpr int kVisReach[kVisClasses] = {3, 4};
// depth: planes per work item along z (the items' z chunks are of that size);
// reach: the stencil class's reach (3 or 4)
template <typename B>
cudaError_t launch_visc_flux(const BoxDev *boxes, const WorkItem *items, int nitems, int depth,
                             int reach, cudaStream_t st);
template <typename B>
cudaError_t launch_update(const BoxDev *boxes, const WorkItem *items, int nitems, int depth,
                          StageArgs sa, bool any_viscous, int reach, cudaStream_t st);

// CRWENO5 / hccs sweeps (crweno_kernels.cu), batched: one work item per tile of
// crweno_tile_lines() lines of one box.  nmax is the longest line among the
// launch's boxes and ms = crweno_segment_rows of it (rows per lane of the
// partitioned line solve); they size the dynamic shared memory.
// sch: SCHEME_CR (crweno5), SCHEME_HC (hccs) or SCHEME_H77 (hccs77); the
// hccs family always solves the bounded system.
cudaError_t prepare_crweno_kernels(bool mixed);
int crweno_tile_lines();
int crweno_lanes(int sch, int n, bool bounded);
int crweno_segment_rows(int sch, int n, bool bounded);
size_t crweno_smem_bytes(int sch, int nmax, int ms, bool mixed);
constexpr int kCrMaxCells = 512;  // longest CRWENO5 / hccs line (shared-memory bound)
// prim_mode (dir 0 only; the blocks own whole x lines): as launch_inviscid's
template <typename B>
cudaError_t launch_crweno(int sch, int dir, const BoxDev *boxes, const WorkItem *items,
                          int nitems, int in_slot, int accumulate, int nmax, int ms,
                          int prim_mode, cudaStream_t st);

}  // namespace nuc3d
