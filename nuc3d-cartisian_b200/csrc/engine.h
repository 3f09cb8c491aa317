// Engine: the host side of the batched solver.  Owns the boxes' device
// memory, the device box table, the per-kernel work-item lists and a CUDA
// graph of one TVD-RK3 step of every active box.  Internal; nuc3d_ctx and
// nuc3d_batch in the C ABI are thin handles over it.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "nuc3d_b200.h"
#include "rhs_kernels.h"

namespace nuc3d {

struct EngineBox {
    nuc3d_box_desc desc{};
    BoxDev dev{};          // host copy of the box's table entry
    int prim_off = 0, prim_n = 0;  // the box's k_prim work items (set by rebuild)
    void *mem = nullptr;   // one stream-ordered allocation holding all fields
    void *force_mem = nullptr;  // spectral forcing scratch (forced boxes only)
    double cfl = 0.5;
    long long steps = 0;   // host mirror of the device step counter
    bool live = false;     // slot in use
};

class Engine {
public:
    Engine(int precision, cudaStream_t stream);
    ~Engine();

    // Adds a box (allocates its device memory, stream-ordered); returns slot id.
    int add_box(const nuc3d_box_desc &d, int *id);
    int remove_box(int id);
    int set_active(int id, bool on);
    int set_cfl(int id, double cfl);
    // host transfers in the device's copy lanes (see chained_host_copy)
    bool copy_lane = false;
    int set_state(int id, const double *const q[5], cudaMemcpyKind kind, bool sync);
    int get_state(int id, double *const q[5], cudaMemcpyKind kind, bool sync);
    // nsteps TVD-RK3 steps of every active box (graph replay unless profiling)
    int step(int nsteps);
    // dt / residual history of the last `n` steps of box id into host arrays
    int history(int id, int n, double *h_dt, double *h_res);
    int rhs(int id, double *const d_rhs[5], double *h_dt_local);
    // Initial state of box id generated on the device (Taylor-Green or HIT);
    // info (may be null): u_rms, Taylor microscale, Reynolds number.  A HIT
    // request with re_lambda > 0 also sets the box's Reynolds number.
    int init_state(int id, const nuc3d_init_desc &in, double info[3]);
    // Turbulence statistics of box id's current state (NUC3D_STATS values).
    int stats(int id, double out[26]);
    // the nine shell spectra of box id into out[9 * kmax] (host); *kmax_out
    // receives kmax = min(nx, ny, nz)/2.  out may be NULL to query kmax.
    int spectra(int id, double *out, int *kmax_out);
    int sync_and_check(int id_or_all);
    double time(int id);
    long long box_steps(int id) const;
    double reynolds(int id) const {
        return id >= 0 && id < (int)boxes_.size() && boxes_[id].live ? boxes_[id].dev.p.reynolds : 0.0;
    }
    int nboxes() const { return (int)boxes_.size(); }
    int precision() const { return precision_; }
    cudaStream_t stream() const { return stream_; }

    // accounting
    long long launches = 0;
    long long graph_captures = 0;  // step graphs captured (one per membership change)
    bool prof_on = false;
    double prof_ms[NUC3D_PROF_CLASSES] = {};
    long long prof_n[NUC3D_PROF_CLASSES] = {};
    int profile_flush();
    // autotuned sweep variant (tile length and run length, kInvTileCells /
    // kInvRunLen) per [scheme JS/Z/-/W7][dir] (-1: not tuned yet) and the
    // measured milliseconds per launch of each variant
    int inv_variant[kSchemes][3] = {{-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1},
                                    {-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1},
                                    {-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1}};
    double inv_tune_ms[kSchemes][3][kInvVariants] = {};
    // autotuned pencil depth of the 2.5-D stencil kernels: index into
    // kPencilDepths (-1: not tuned yet), the measured milliseconds of one
    // viscous-flux + update pass per depth, and the active cells it was tuned
    // at (a batch that grows or shrinks past 2x is tuned again)
    int pencil_variant = -1;
    double pencil_tune_ms[3] = {};
    long long pencil_tuned_cells = 0;

    static long long box_bytes(const nuc3d_box_desc &d);
    static int validate(const nuc3d_box_desc &d, std::string *why);

private:
    // issues this engine's copies of a host<->device state transfer (dir 0:
    // upload, 1: download) after the last such transfer any engine on the
    // device issued in that direction (copy lanes, engine.cu)
    int chained_host_copy(int dir, int id, double *const host[5]);
    int rebuild();
    // launches of one step into stream s (eager on stream_, or on the private
    // capture stream while recording the graph)
    int enqueue_step(cudaStream_t s);
    template <typename B>
    int enqueue_step_t(cudaStream_t s);
    template <typename B>
    int enqueue_rhs_t(int id, double *const d_rhs[5]);
    template <typename B>
    cudaError_t enqueue_forcing(cudaStream_t st);
    // the 2.5-D kernels of both stencil classes at pencil-depth variant v
    template <typename B>
    cudaError_t launch_visc_classes(int v, cudaStream_t st);
    template <typename B>
    cudaError_t launch_update_classes(int v, StageArgs sa, cudaStream_t st);
    void invalidate_graph();
    int autotune();

    int precision_;
    cudaStream_t stream_;
    std::vector<EngineBox> boxes_;
    bool dirty_ = true;
    bool any_visc_ = false;
    int nactive_ = 0;
    BoxDev *d_boxes_ = nullptr;
    int d_boxes_cap_ = 0;
    WorkItem *d_items_ = nullptr;
    size_t d_items_cap_ = 0;
    // offsets/counts into d_items_
    struct Range {
        size_t off = 0;
        int n = 0;
    };
    Range r_prim_;
    Range r_inv_[kSchemes][3][kInvTileClasses];  // [scheme id][dir][32/64-cell tiles]
    // the work list of the variant the autotuner chose (32-cell tiles before)
    const Range &inv_range(int s, int d) const {
        return r_inv_[s][d][inv_variant[s][d] < 0 ? 0 : inv_tile_class(inv_variant[s][d])];
    }
    // 2.5-D stencil tiles per [stencil class (kVisReach)][pencil depth of
    // kPencilDepths]
    Range r_25d_[kVisClasses][3];
    long long active_cells_ = 0;
    int pv() const { return pencil_variant < 0 ? 0 : pencil_variant; }
    // Mixed precision stages each line's split fluxes as FP32 offsets from
    // their value at the tile's first cell, so the rounding depends on where
    // tiles start: only the 32-cell tiles run there, which keeps every
    // variant (and a box alone or in any batch) bitwise the same.
    bool mixed_tiles_only32() const { return precision_ == NUC3D_MIXED; }
    // line-solve tiles per [line scheme: 0 crweno5, 1 hccs, 2 hccs77][dir],
    // with the longest line and the rows per lane that size each launch's
    // shared memory
    Range r_cr_[kLineSchemes][3];
    int cr_nmax_[kLineSchemes][3] = {}, cr_ms_[kLineSchemes][3] = {};
    int launches_per_step_ = 0;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
    cudaStream_t cap_stream_ = nullptr;  // graphs cannot be captured on the legacy stream
    cudaStream_t fork_stream_ = nullptr;  // the captured step's viscous-flux branch
    cudaEvent_t fork_ev_[2] = {nullptr, nullptr};  // fork after the x sweep, join before the update
    unsigned *h_flags_ = nullptr;      // mapped page-locked mirror of the boxes' flags
    unsigned *h_flags_dev_ = nullptr;  // its device address
    int h_flags_cap_ = 0;
    int device_ = 0;                      // the device current at construction
    cudaEvent_t copy_ev_[2] = {nullptr, nullptr};  // this engine's last upload / download
    double **d_rhs_ptrs_ = nullptr;  // 5 per box, for stage -1
    double *d_stats_ = nullptr;       // statistics scratch
    // profiling events
    std::vector<cudaEvent_t> ev_pool_;
    struct Mark {
        int cls;
        cudaEvent_t a, b;
    };
    std::vector<Mark> pending_;
    size_t ev_next_ = 0;
    friend struct ProfScope;
};

}  // namespace nuc3d
