// Engine: host side of the batched solver (see engine.h).
#include "engine.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>

#include "forcing_kernels.h"
#include "init_kernels.h"
#include "spectra_kernels.h"
#include "stats_kernels.h"
#include "op_kernels.h"

namespace nuc3d {

namespace {

long long pad32(long long n) { return (n + 31) / 32 * 32; }
size_t bulk_size(int precision) { return precision == NUC3D_MIXED ? sizeof(float) : sizeof(double); }
// the box's small area: eig, residual sum, flags, StepScalars, then the
// viscous-flux kernel's 8 TMA tensor maps (128-byte aligned)
constexpr size_t kTmaOff = (256 + sizeof(StepScalars) + 127) / 128 * 128;
constexpr size_t kSmallBytes = kTmaOff + 8 * sizeof(CUtensorMap);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when unavailable
PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// Tensor maps of u, v, w, T for k_visc_flux25's TMA loads: [0..3] the tile's
// plane with its halo (kViscTmaHaloX x kViscTmaHaloY), [4..7] the tile's own
// columns (kViscTmaTileX x kViscTmaTileY), one plane deep.  A row must be a
// multiple of 16 bytes (nx even); NUC3D_VISC_TMA=0 keeps the element-wise
// cp.async loads for every tile.
bool encode_visc_maps(const BoxDev &d, CUtensorMap out[8]) {
    const BoxParams &p = d.p;
    if (p.n[0] % 2 != 0) return false;
    if (const char *env = std::getenv("NUC3D_VISC_TMA"))
        if (std::atoi(env) == 0) return false;
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tma_encoder();
    if (!enc) return false;
    const int src[4] = {0, 1, 2, 5};  // u, v, w, T
    const cuuint64_t dims[3] = {(cuuint64_t)p.n[0], (cuuint64_t)p.n[1], (cuuint64_t)p.n[2]};
    const cuuint64_t strides[2] = {(cuuint64_t)p.stride[1] * 8, (cuuint64_t)p.stride[2] * 8};
    const cuuint32_t es[3] = {1, 1, 1};
    for (int kind = 0; kind < 2; ++kind) {
        const cuuint32_t box[3] = {(cuuint32_t)(kind ? kViscTmaTileX : kViscTmaHaloX),
                                   (cuuint32_t)(kind ? kViscTmaTileY : kViscTmaHaloY), 1};
        for (int f = 0; f < 4; ++f) {
            CUresult r = enc(&out[4 * kind + f], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                             static_cast<void *>(fieldW(d, src[f])), dims, strides, box, es,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return false;
        }
    }
    return true;
}

BoxParams make_params(const nuc3d_box_desc &d) {
    BoxParams bp{};
    bp.n[0] = d.nx;
    bp.n[1] = d.ny;
    bp.n[2] = d.nz;
    bp.N = (long long)d.nx * d.ny * d.nz;
    bp.stride[0] = 1;
    bp.stride[1] = d.nx;
    bp.stride[2] = (long long)d.nx * d.ny;
    bp.d[0] = d.lx / d.nx;  // block.cpp:62-64
    bp.d[1] = d.ly / d.ny;
    bp.d[2] = d.lz / d.nz;
    for (int i = 0; i < 3; ++i) bp.inv_d[i] = 1.0 / bp.d[i];
    bp.gamma = d.gamma;
    bp.mach = d.mach;
    bp.reynolds = d.reynolds;
    bp.prandtl = d.prandtl;
    bp.tref_nd = d.t_ref / d.t_inf;
    bp.powerlaw_exp = d.powerlaw_exp;
    bp.cfl = 0.5;
    bp.visc_model = d.visc_model;
    bp.navier_stokes = d.pde_model == NUC3D_NAVIERSTOKES3D;
    bp.quirks = d.quirks;
    for (int i = 0; i < 3; ++i) bp.scheme[i] = d.scheme[i];
    bp.riemann = d.riemann;
    // differential schemes as coefficients of f(i+m) - f(i-m), m = 1..4
    // (schemes.hpp:36-42)
    for (int i = 0; i < 3; ++i) {
        bp.vis[i] = d.vis_scheme[i];
        double *c = bp.vcoef[i];
        c[0] = c[1] = c[2] = c[3] = 0.0;
        if (d.vis_scheme[i] == NUC3D_CD2) {
            c[0] = K::C21;
        } else if (d.vis_scheme[i] == NUC3D_CD8) {
            c[0] = K::C81, c[1] = K::C82, c[2] = K::C83, c[3] = K::C84;
        } else {
            c[0] = K::CD1, c[1] = K::CD2, c[2] = K::CD3;
        }
    }
    return bp;
}

// stencil class of the 2.5-D kernels (kVisReach): 1 for a Navier-Stokes box
// with cd2 or cd8 in some direction
int vis_class(const BoxParams &p) {
    return p.navier_stokes && (p.vis[0] != VIS_CD6 || p.vis[1] != VIS_CD6 || p.vis[2] != VIS_CD6)
               ? 1
               : 0;
}

int ceil_div(int a, int b) { return (a + b - 1) / b; }

}  // namespace

#define ECK(call)                                                         \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) {                                          \
            set_last_error(NUC3D_ERR_CUDA, (std::string(#call) + ": " +   \
                                            cudaGetErrorString(e_)).c_str()); \
            return NUC3D_ERR_CUDA;                                        \
        }                                                                 \
    } while (0)

int Engine::validate(const nuc3d_box_desc &d, std::string *why) {
    auto bad = [&](int code, const char *m) {
        if (why) *why = m;
        return code;
    };
    const int n[3] = {d.nx, d.ny, d.nz};
    for (int i = 0; i < 3; ++i) {
        if (n[i] < 8) return bad(NUC3D_ERR_INVALID, "every box extent must be >= 8 cells");
        if (d.scheme[i] < NUC3D_WENO5JS || d.scheme[i] > NUC3D_UPWIND1ST)
            return bad(NUC3D_ERR_UNSUPPORTED, "unknown reconstruction scheme");
    }
    for (int i = 0; i < 3; ++i)
        if (line_slot(d.scheme[i]) >= 0 && n[i] > kCrMaxCells)
            return bad(NUC3D_ERR_UNSUPPORTED, "CRWENO5 / hccs / hccs77 lines are limited to 512 cells");
    for (int i = 0; i < 3; ++i)
        if ((d.scheme[i] == NUC3D_HCCS || d.scheme[i] == NUC3D_HCCS77) && n[i] < 9)
            return bad(NUC3D_ERR_INVALID, "hccs / hccs77 lines need at least 9 cells");
    if ((long long)d.nx * d.ny * d.nz > (1LL << 31)) return bad(NUC3D_ERR_INVALID, "box larger than 2^31 cells");
    if (!(d.lx > 0 && d.ly > 0 && d.lz > 0)) return bad(NUC3D_ERR_INVALID, "box lengths must be > 0");
    if (d.pde_model != NUC3D_EULER3D && d.pde_model != NUC3D_NAVIERSTOKES3D)
        return bad(NUC3D_ERR_UNSUPPORTED, "unknown PDE model");
    if (d.visc_model < NUC3D_VISC_SUTHERLAND || d.visc_model > NUC3D_VISC_POWERLAW)
        return bad(NUC3D_ERR_UNSUPPORTED, "unknown viscosity model");
    if (d.precision != NUC3D_FP64 && d.precision != NUC3D_MIXED)
        return bad(NUC3D_ERR_UNSUPPORTED, "unknown precision");
    if (!(d.gamma > 1.0) || !(d.mach > 0.0) || !(d.reynolds > 0.0) || !(d.prandtl > 0.0))
        return bad(NUC3D_ERR_INVALID, "gamma must be > 1 and Mach, Re, Pr > 0");
    if (d.riemann < NUC3D_RIEMANN_LF || d.riemann > NUC3D_RIEMANN_AUSMP)
        return bad(NUC3D_ERR_UNSUPPORTED, "unknown Riemann solver (flux splitting)");
    for (int i = 0; i < 3; ++i)
        if (d.vis_scheme[i] < NUC3D_CD6 || d.vis_scheme[i] > NUC3D_CD8)
            return bad(NUC3D_ERR_UNSUPPORTED, "unknown differential scheme");
    if (d.forcing != NUC3D_FORCING_NONE && d.forcing != NUC3D_FORCING_CONST &&
        d.forcing != NUC3D_FORCING_BAND)
        return bad(NUC3D_ERR_UNSUPPORTED, "unknown forcing model");
    if (d.forcing != NUC3D_FORCING_NONE) {
        if (!(d.forcing_k > 0.0) || forcing_K(d.forcing_k) > kForceMaxK)
            return bad(NUC3D_ERR_UNSUPPORTED, "forcing shell radius must be in (0, 3.5)");
        if (d.forcing == NUC3D_FORCING_BAND && !(d.forcing_amp >= 0.0))
            return bad(NUC3D_ERR_INVALID, "band forcing needs an injection rate >= 0");
        for (int i = 0; i < 3; ++i)
            if (2 * forcing_K(d.forcing_k) + 1 > n[i])
                return bad(NUC3D_ERR_INVALID, "box too small for the forcing shell");
    }
    return NUC3D_OK;
}

long long Engine::box_bytes(const nuc3d_box_desc &d) {
    if (validate(d, nullptr) != NUC3D_OK) return -1;
    BoxParams bp = make_params(d);
    long long np = pad32(bp.N);
    long long bs = (long long)bulk_size(d.precision);
    long long b = 21 * np * 8 + 14 * np * bs + (long long)kSmallBytes;
    if (d.forcing != NUC3D_FORCING_NONE) b += (long long)forcing_scratch_bytes(bp, d.forcing_k);
    return b;
}

namespace {
// Copy lanes.  Host<->device state transfers of the engines on a device that
// have their copy lane on run one at a time per direction, in submission
// order (a transfer waits for the previously submitted one, whatever that
// one waits for on its own stream): two large transfers in
// flight in the same direction share the host link and both finish late, and
// so do the steps that wait on them (at 256^3, two 671 MB uploads issued
// together took 27 ms each against 12 ms one after the other).  Chained, each
// transfer has the whole link; uploads and downloads still overlap each other
// and the steps of other engines.  A lane holds the event of the last
// transfer and the engine that owns it.
struct CopyLane {
    const void *owner = nullptr;
    cudaEvent_t ev = nullptr;
};
std::mutex g_lane_mu;
std::map<int, CopyLane> g_lanes[2];  // [upload, download][device]

// NUC3D_STEP_FORK=0 keeps a captured step on one stream (the viscous fluxes
// then run between the x and y sweeps); the default forks them
bool step_fork_enabled() {
    const char *env = std::getenv("NUC3D_STEP_FORK");
    return !(env && env[0] == '0');
}

// the flags pointers of up to kMax boxes, passed by value to k_export_flags
struct FlagPtrs {
    static constexpr int kMax = 32;
    const unsigned *p[kMax];
    int n;
};
// flags of up to kMax boxes -> mapped host memory (zero-copy stores)
__global__ void k_export_flags(FlagPtrs f, unsigned *out) {
    const int i = threadIdx.x;
    if (i < f.n) out[i] = *f.p[i];
}
}  // namespace

Engine::Engine(int precision, cudaStream_t stream) : precision_(precision), stream_(stream) {
    cudaGetDevice(&device_);
}

Engine::~Engine() {
    {
        std::lock_guard<std::mutex> lk(g_lane_mu);
        for (auto &lanes : g_lanes) {
            auto it = lanes.find(device_);
            if (it != lanes.end() && it->second.owner == this) it->second = CopyLane{};
        }
    }
    cudaStreamSynchronize(stream_);
    invalidate_graph();
    for (auto &b : boxes_) {
        if (b.mem) cudaFreeAsync(b.mem, stream_);
        if (b.force_mem) cudaFreeAsync(b.force_mem, stream_);
    }
    if (d_boxes_) cudaFreeAsync(d_boxes_, stream_);
    if (d_items_) cudaFreeAsync(d_items_, stream_);
    if (d_rhs_ptrs_) cudaFreeAsync(d_rhs_ptrs_, stream_);
    if (d_stats_) cudaFreeAsync(d_stats_, stream_);
    cudaStreamSynchronize(stream_);
    for (cudaEvent_t e : ev_pool_) cudaEventDestroy(e);
    for (cudaEvent_t e : copy_ev_)
        if (e) cudaEventDestroy(e);
    if (h_flags_) cudaFreeHost(h_flags_);
    if (cap_stream_) cudaStreamDestroy(cap_stream_);
    if (fork_stream_) cudaStreamDestroy(fork_stream_);
    for (cudaEvent_t e : fork_ev_)
        if (e) cudaEventDestroy(e);
}

void Engine::invalidate_graph() {
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    exec_ = nullptr;
    graph_ = nullptr;
}

int Engine::add_box(const nuc3d_box_desc &d, int *id) {
    std::string why;
    int rc = validate(d, &why);
    if (rc) return set_last_error(rc, why.c_str());
    if (d.precision != precision_)
        return set_last_error(NUC3D_ERR_INVALID, "box precision differs from the batch's");
    EngineBox b;
    b.desc = d;
    b.dev.p = make_params(d);
    const long long np = pad32(b.dev.p.N);
    const size_t bs = bulk_size(precision_);
    const size_t bytes = sizeof(double) * 21 * (size_t)np + bs * 14 * (size_t)np + kSmallBytes;
    cudaError_t e = cudaMallocAsync(&b.mem, bytes, stream_);
    if (e == cudaSuccess && d.forcing != NUC3D_FORCING_NONE)
        e = cudaMallocAsync(&b.force_mem, forcing_scratch_bytes(b.dev.p, d.forcing_k), stream_);
    if (e != cudaSuccess) {
        if (b.mem) cudaFreeAsync(b.mem, stream_);
        cudaGetLastError();
        return set_last_error(NUC3D_ERR_NOMEM,
                              (std::string("device allocation failed: ") + cudaGetErrorString(e)).c_str());
    }
    double *dp = static_cast<double *>(b.mem);
    b.dev.base = dp;
    b.dev.np = np;
    char *bk = reinterpret_cast<char *>(dp + 21 * (size_t)np);
    char *sm = bk + bs * 14 * (size_t)np;
    b.dev.eig = reinterpret_cast<double *>(sm);
    b.dev.res_acc = reinterpret_cast<double *>(sm + 64);
    b.dev.flags = reinterpret_cast<unsigned *>(sm + 128);
    b.dev.sc = reinterpret_cast<StepScalars *>(sm + 256);
    b.dev.active = 1;
    b.live = true;
    ECK(cudaMemsetAsync(b.mem, 0, bytes, stream_));
    // sc->cfl = 0.5 (the stream-ordered memset above runs first)
    static const double half = 0.5;
    ECK(cudaMemcpyAsync(&b.dev.sc->cfl, &half, sizeof half, cudaMemcpyHostToDevice, stream_));
    if (b.force_mem)
        ECK(forcing_prepare(b.dev.p, d.forcing_k, forcing_layout(b.dev.p, d.forcing_k, b.force_mem),
                            stream_));
    b.dev.tmw = nullptr;
    if (b.dev.p.navier_stokes) {
        CUtensorMap maps[8];
        if (encode_visc_maps(b.dev, maps)) {
            void *dst = sm + kTmaOff;
            ECK(cudaMemcpyAsync(dst, maps, sizeof maps, cudaMemcpyHostToDevice, stream_));
            ECK(cudaStreamSynchronize(stream_));  // maps is a host stack array
            b.dev.tmw = dst;
        }
    }
    int slot = -1;
    for (size_t i = 0; i < boxes_.size(); ++i)
        if (!boxes_[i].live) {
            slot = (int)i;
            break;
        }
    if (slot < 0) {
        slot = (int)boxes_.size();
        boxes_.push_back(b);
    } else {
        boxes_[slot] = b;
    }
    *id = slot;
    dirty_ = true;
    return NUC3D_OK;
}

int Engine::remove_box(int id) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live)
        return set_last_error(NUC3D_ERR_INVALID, "no such box");
    EngineBox &b = boxes_[id];
    ECK(cudaFreeAsync(b.mem, stream_));
    if (b.force_mem) ECK(cudaFreeAsync(b.force_mem, stream_));
    b = EngineBox();
    dirty_ = true;
    return NUC3D_OK;
}

int Engine::set_active(int id, bool on) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live)
        return set_last_error(NUC3D_ERR_INVALID, "no such box");
    if ((boxes_[id].dev.active != 0) != on) {
        boxes_[id].dev.active = on ? 1 : 0;
        dirty_ = true;
    }
    return NUC3D_OK;
}

int Engine::set_cfl(int id, double cfl) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live)
        return set_last_error(NUC3D_ERR_INVALID, "no such box");
    if (!(cfl > 0.0)) return set_last_error(NUC3D_ERR_INVALID, "cfl must be > 0");
    EngineBox &b = boxes_[id];
    if (b.cfl != cfl) {
        b.cfl = cfl;
        ECK(cudaMemcpyAsync(&b.dev.sc->cfl, &b.cfl, sizeof(double), cudaMemcpyHostToDevice, stream_));
        ECK(cudaStreamSynchronize(stream_));  // b.cfl is the pageable source
    }
    return NUC3D_OK;
}

int Engine::chained_host_copy(int dir, int id, double *const host[5]) {
    EngineBox &b = boxes_[id];
    const size_t bytes = sizeof(double) * (size_t)b.dev.p.N;
    if (!copy_ev_[dir]) ECK(cudaEventCreateWithFlags(&copy_ev_[dir], cudaEventDisableTiming));
    std::lock_guard<std::mutex> lk(g_lane_mu);
    CopyLane &lane = g_lanes[dir][device_];
    // (this engine's own earlier transfers are ordered by its stream)
    if (lane.ev && lane.owner != this) ECK(cudaStreamWaitEvent(stream_, lane.ev, 0));
    for (int e = 0; e < 5; ++e) {
        if (dir == 0)
            ECK(cudaMemcpyAsync(fieldU(b.dev, 0, e), host[e], bytes, cudaMemcpyHostToDevice,
                                stream_));
        else
            ECK(cudaMemcpyAsync(host[e], fieldU(b.dev, 0, e), bytes, cudaMemcpyDeviceToHost,
                                stream_));
    }
    ECK(cudaEventRecord(copy_ev_[dir], stream_));
    lane.owner = this;
    lane.ev = copy_ev_[dir];
    return NUC3D_OK;
}

int Engine::set_state(int id, const double *const q[5], cudaMemcpyKind kind, bool sync) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live)
        return set_last_error(NUC3D_ERR_INVALID, "no such box");
    if (!q) return set_last_error(NUC3D_ERR_INVALID, "null argument");
    for (int e = 0; e < 5; ++e)
        if (!q[e]) return set_last_error(NUC3D_ERR_INVALID, "null field pointer");
    EngineBox &b = boxes_[id];
    size_t bytes = sizeof(double) * (size_t)b.dev.p.N;
    if (kind == cudaMemcpyHostToDevice && copy_lane) {
        int rc = chained_host_copy(0, id, const_cast<double *const *>(q));
        if (rc) return rc;
    } else {
        for (int e = 0; e < 5; ++e)
            ECK(cudaMemcpyAsync(fieldU(b.dev, 0, e), q[e], bytes, kind, stream_));
    }
    if (sync) ECK(cudaStreamSynchronize(stream_));
    return NUC3D_OK;
}

int Engine::get_state(int id, double *const q[5], cudaMemcpyKind kind, bool sync) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live)
        return set_last_error(NUC3D_ERR_INVALID, "no such box");
    if (!q) return set_last_error(NUC3D_ERR_INVALID, "null argument");
    for (int e = 0; e < 5; ++e)
        if (!q[e]) return set_last_error(NUC3D_ERR_INVALID, "null field pointer");
    EngineBox &b = boxes_[id];
    size_t bytes = sizeof(double) * (size_t)b.dev.p.N;
    if (kind == cudaMemcpyDeviceToHost && copy_lane) {
        int rc = chained_host_copy(1, id, q);
        if (rc) return rc;
    } else {
        for (int e = 0; e < 5; ++e)
            ECK(cudaMemcpyAsync(q[e], fieldU(b.dev, 0, e), bytes, kind, stream_));
    }
    if (sync) ECK(cudaStreamSynchronize(stream_));
    return NUC3D_OK;
}

int Engine::rebuild() {
    invalidate_graph();
    ECK(cudaStreamSynchronize(stream_));
    const bool mixed = precision_ == NUC3D_MIXED;
    std::vector<BoxDev> table(boxes_.size());
    std::vector<WorkItem> prim, st25[kVisClasses][3], inv[kSchemes][3][kInvTileClasses],
        cr[kLineSchemes][3];
    const int crtl = crweno_tile_lines();
    for (int c = 0; c < kLineSchemes; ++c)
        for (int d = 0; d < 3; ++d) cr_nmax_[c][d] = cr_ms_[c][d] = 0;
    any_visc_ = false;
    nactive_ = 0;
    active_cells_ = 0;
    for (size_t i = 0; i < boxes_.size(); ++i) {
        EngineBox &b = boxes_[i];
        table[i] = b.dev;
        if (!b.live) table[i].active = 0;
        if (!b.live || !b.dev.active) continue;
        ++nactive_;
        const BoxParams &p = b.dev.p;
        active_cells_ += p.N;
        const int id = (int)i;
        any_visc_ = any_visc_ || p.navier_stokes;
        boxes_[i].prim_off = (int)prim.size();
        for (long long c = 0; c * kPrimChunk < p.N; ++c)
            prim.push_back({id, (int)c, (int)std::min<long long>(kPrimChunk, p.N - c * kPrimChunk), 0});
        boxes_[i].prim_n = (int)prim.size() - boxes_[i].prim_off;
        const int vc = vis_class(p);
        for (int v = 0; v < 3; ++v)
            for (int z = 0; z < ceil_div(p.n[2], kPencilDepths[v]); ++z)
                for (int y = 0; y < ceil_div(p.n[1], kT25Y); ++y)
                    for (int x = 0; x < ceil_div(p.n[0], kT25X); ++x)
                        st25[vc][v].push_back({id, x, y, z});
        for (int d = 0; d < 3; ++d) {
            int s = p.scheme[d];
            if (line_slot(s) >= 0) {
                const int c = line_slot(s);
                const bool bounded = s != SCHEME_CR || (p.quirks & QK_CRWENO_BOUNDED) != 0;
                cr_nmax_[c][d] = std::max(cr_nmax_[c][d], p.n[d]);
                cr_ms_[c][d] = std::max(cr_ms_[c][d], crweno_segment_rows(s, p.n[d], bounded));
                auto &L = cr[c][d];
                if (d == 0) {
                    for (int k = 0; k < p.n[2]; ++k)
                        for (int g = 0; g < ceil_div(p.n[1], crtl); ++g) L.push_back({id, g, k, 0});
                } else if (d == 1) {
                    for (int k = 0; k < p.n[2]; ++k)
                        for (int g = 0; g < ceil_div(p.n[0], crtl); ++g) L.push_back({id, g, k, 0});
                } else {
                    for (int j = 0; j < p.n[1]; ++j)
                        for (int g = 0; g < ceil_div(p.n[0], crtl); ++g) L.push_back({id, g, j, 0});
                }
                continue;
            }
            for (int tc = 0; tc < kInvTileClasses; ++tc) {
                InvTileDims t = inviscid_tile(d, mixed, tc == 0 ? 32 : 64);
                auto &L = inv[s][d][tc];
                if (d == 0) {
                    for (int k = 0; k < p.n[2]; ++k)
                        for (int b2 = 0; b2 < ceil_div(p.n[1], t.TL); ++b2)
                            for (int a = 0; a < ceil_div(p.n[0], t.TC); ++a) L.push_back({id, a, b2, k});
                } else if (d == 1) {
                    for (int k = 0; k < p.n[2]; ++k)
                        for (int b2 = 0; b2 < ceil_div(p.n[1], t.TC); ++b2)
                            for (int a = 0; a < ceil_div(p.n[0], t.TL); ++a) L.push_back({id, a, b2, k});
                } else {
                    for (int c = 0; c < ceil_div(p.n[2], t.TC); ++c)
                        for (int j = 0; j < p.n[1]; ++j)
                            for (int a = 0; a < ceil_div(p.n[0], t.TL); ++a) L.push_back({id, a, j, c});
                }
            }
        }
    }
    std::vector<WorkItem> all;
    auto append = [&](const std::vector<WorkItem> &v, Range &r) {
        r.off = all.size();
        r.n = (int)v.size();
        all.insert(all.end(), v.begin(), v.end());
    };
    append(prim, r_prim_);
    for (int c = 0; c < kVisClasses; ++c)
        for (int v = 0; v < 3; ++v) append(st25[c][v], r_25d_[c][v]);
    for (int s = 0; s < kSchemes; ++s)
        for (int d = 0; d < 3; ++d)
            for (int tc = 0; tc < kInvTileClasses; ++tc) append(inv[s][d][tc], r_inv_[s][d][tc]);
    for (int c = 0; c < kLineSchemes; ++c)
        for (int d = 0; d < 3; ++d) append(cr[c][d], r_cr_[c][d]);
    if ((int)boxes_.size() > d_boxes_cap_) {
        if (d_boxes_) ECK(cudaFreeAsync(d_boxes_, stream_));
        if (d_rhs_ptrs_) ECK(cudaFreeAsync(d_rhs_ptrs_, stream_));
        d_boxes_cap_ = std::max<int>(8, (int)boxes_.size() * 2);
        ECK(cudaMallocAsync(&d_boxes_, sizeof(BoxDev) * d_boxes_cap_, stream_));
        ECK(cudaMallocAsync(&d_rhs_ptrs_, sizeof(double *) * 5 * d_boxes_cap_, stream_));
    }
    if (all.size() > d_items_cap_) {
        if (d_items_) ECK(cudaFreeAsync(d_items_, stream_));
        d_items_cap_ = std::max<size_t>(1024, all.size() * 5 / 4);
        ECK(cudaMallocAsync(&d_items_, sizeof(WorkItem) * d_items_cap_, stream_));
    }
    if (!table.empty())
        ECK(cudaMemcpyAsync(d_boxes_, table.data(), sizeof(BoxDev) * table.size(),
                            cudaMemcpyHostToDevice, stream_));
    if (!all.empty())
        ECK(cudaMemcpyAsync(d_items_, all.data(), sizeof(WorkItem) * all.size(),
                            cudaMemcpyHostToDevice, stream_));
    ECK(cudaStreamSynchronize(stream_));  // host vectors go out of scope
    ECK(prepare_inviscid_kernels(mixed));
    ECK(prepare_crweno_kernels(mixed));
    ECK(prepare_stencil_kernels(mixed));
    int per_stage = 0;
    for (int c = 0; c < kVisClasses; ++c)
        per_stage += (any_visc_ && r_25d_[c][0].n > 0) + (r_25d_[c][0].n > 0);
    for (int s = 0; s < kSchemes; ++s)
        for (int d = 0; d < 3; ++d) per_stage += r_inv_[s][d][0].n > 0;
    for (int c = 0; c < kLineSchemes; ++c)
        for (int d = 0; d < 3; ++d) per_stage += r_cr_[c][d].n > 0;
    launches_per_step_ = 3 * per_stage + 3;  // + clear_eig, dt, residual
    for (const EngineBox &b : boxes_)
        if (b.live && b.dev.active && b.force_mem) launches_per_step_ += 3 * 8;  // forcing passes
    dirty_ = false;
    return NUC3D_OK;
}

// Kernel-class timing while profiling (eager launches only).
struct ProfScope {
    Engine *e;
    int cls;
    cudaEvent_t a = nullptr;
    cudaEvent_t get() {
        if (e->ev_next_ == e->ev_pool_.size()) {
            cudaEvent_t ev;
            if (cudaEventCreate(&ev) != cudaSuccess) return nullptr;
            e->ev_pool_.push_back(ev);
        }
        return e->ev_pool_[e->ev_next_++];
    }
    ProfScope(Engine *e_, int cls_) : e(e_), cls(cls_) {
        if (e->prof_on && (a = get())) cudaEventRecord(a, e->stream_);
    }
    ~ProfScope() {
        if (!a) return;
        cudaEvent_t b = get();
        if (!b) return;
        cudaEventRecord(b, e->stream_);
        e->pending_.push_back({cls, a, b});
    }
};

int Engine::profile_flush() {
    if (pending_.empty()) return NUC3D_OK;
    ECK(cudaStreamSynchronize(stream_));
    for (auto &m : pending_) {
        float ms = 0.f;
        ECK(cudaEventElapsedTime(&ms, m.a, m.b));
        prof_ms[m.cls] += ms;
        prof_n[m.cls] += 1;
    }
    pending_.clear();
    ev_next_ = 0;
    return NUC3D_OK;
}

template <typename B>
int Engine::enqueue_step_t(cudaStream_t st) {
    const int nb = (int)boxes_.size();
    const WorkItem *it = d_items_;
    {
        ProfScope ps(this, NUC3D_PROF_DT);
        ECK(launch_clear_eig(d_boxes_, nb, st));
    }
    for (int stage = 0; stage < 3; ++stage) {
        const int in = stage, out = (stage + 1) % 3;
        // the x sweeps (WENO tiles and CRWENO5 / hccs lines alike) recover
        // the primitives of their cells, and on the first stage fold the
        // eigenvalue maxima, before their splits
        auto sweeps = [&](int d) -> int {
            ProfScope ps(this, NUC3D_PROF_INV_X + d);
            const int prim_mode = d == 0 ? (stage == 0 ? 2 : 1) : 0;
            for (int s = 0; s < kSchemes; ++s)
                ECK((launch_inviscid<B>(s, d, inv_variant[s][d], d_boxes_, it + inv_range(s, d).off,
                                        inv_range(s, d).n, in, d > 0, prim_mode, st)));
            for (int c = 0; c < kLineSchemes; ++c)
                ECK((launch_crweno<B>(kLineScheme[c], d, d_boxes_,
                                      it + r_cr_[c][d].off, r_cr_[c][d].n, in, d > 0,
                                      cr_nmax_[c][d], cr_ms_[c][d], prim_mode, st)));
            return NUC3D_OK;
        };
        if (int rc = sweeps(0)) return rc;
        if (stage == 0) {
            ProfScope ps(this, NUC3D_PROF_DT);
            ECK(launch_dt(d_boxes_, nb, st));
        }
        // The viscous fluxes need only this stage's primitives (the x sweep)
        // and only the update reads them: in a captured step they run on a
        // forked stream, beside the y and z sweeps (an HBM- and
        // latency-bound kernel next to FP64-bound ones), and join before the
        // update.  Eager (profiled) steps keep one stream.
        const bool fork = any_visc_ && fork_stream_ && st == cap_stream_;
        if (any_visc_) {
            ProfScope ps(this, NUC3D_PROF_VISC);
            cudaStream_t vs = st;
            if (fork) {
                ECK(cudaEventRecord(fork_ev_[0], st));
                ECK(cudaStreamWaitEvent(fork_stream_, fork_ev_[0], 0));
                vs = fork_stream_;
            }
            ECK(launch_visc_classes<B>(pv(), vs));
            if (fork) ECK(cudaEventRecord(fork_ev_[1], fork_stream_));
        }
        for (int d = 1; d < 3; ++d)
            if (int rc = sweeps(d)) return rc;
        ECK(enqueue_forcing<B>(st));
        if (fork) ECK(cudaStreamWaitEvent(st, fork_ev_[1], 0));
        {
            ProfScope ps(this, NUC3D_PROF_UPDATE);
            StageArgs sa{stage, in, out, nullptr};
            ECK(launch_update_classes<B>(pv(), sa, st));
        }
    }
    {
        ProfScope ps(this, NUC3D_PROF_RESIDUAL);
        ECK(launch_residual(d_boxes_, nb, st));
    }
    return NUC3D_OK;
}

template <typename B>
cudaError_t Engine::launch_visc_classes(int v, cudaStream_t st) {
    for (int c = 0; c < kVisClasses; ++c) {
        const Range &rg = r_25d_[c][v];
        cudaError_t e = launch_visc_flux<B>(d_boxes_, d_items_ + rg.off, rg.n, kPencilDepths[v],
                                            kVisReach[c], st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <typename B>
cudaError_t Engine::launch_update_classes(int v, StageArgs sa, cudaStream_t st) {
    for (int c = 0; c < kVisClasses; ++c) {
        const Range &rg = r_25d_[c][v];
        cudaError_t e = launch_update<B>(d_boxes_, d_items_ + rg.off, rg.n, kPencilDepths[v], sa,
                                         any_visc_, kVisReach[c], st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Spectral forcing of the forced boxes (physicsModel::solveSource after
// the RHS assembly, NaiverStokes3d.cpp:58): uses this stage's primitives W,
// subtracts from the inviscid accumulator R before the update.
template <typename B>
cudaError_t Engine::enqueue_forcing(cudaStream_t st) {
    for (const EngineBox &b : boxes_) {
        if (!b.live || !b.dev.active || !b.force_mem) continue;
        ForceParams fp{b.desc.forcing_amp, b.desc.forcing_hel, b.desc.forcing_k,
                       forcing_K(b.desc.forcing_k), b.desc.forcing == NUC3D_FORCING_BAND ? 1 : 0};
        cudaError_t e = launch_forcing<B>(b.dev, forcing_layout(b.dev.p, b.desc.forcing_k, b.force_mem),
                                          fp, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int Engine::enqueue_step(cudaStream_t s) {
    return precision_ == NUC3D_MIXED ? enqueue_step_t<float>(s) : enqueue_step_t<double>(s);
}

// Picks the run length of the directional sweep per scheme and direction,
// and the pencil depth of the 2.5-D stencil kernels, by timing every variant
// on this batch's own work lists: the sweeps on the first step after a
// rebuild that brings a new (scheme, direction) pair, the depth on the first
// step and whenever the active cells have moved past 2x (or 1/2x) of those
// it was tuned at.  The sweeps only write the RHS accumulator (and the x
// sweep the primitives, with the values they already hold) and the
// viscous-flux kernel the viscous fluxes, which every stage recomputes; the
// update is timed as a first stage, which writes only the u1 slot that the
// next step's first stage overwrites (and no residual), so timing on the
// live state changes nothing.
int Engine::autotune() {
    bool need_sweep = false;
    for (int s = 0; s < kSchemes; ++s)
        for (int d = 0; d < 3; ++d)
            need_sweep = need_sweep || (r_inv_[s][d][0].n > 0 && inv_variant[s][d] < 0);
    const bool need_pencil =
        (r_25d_[0][0].n > 0 || r_25d_[1][0].n > 0) &&
        (pencil_variant < 0 || 2 * active_cells_ < pencil_tuned_cells ||
                            active_cells_ > 2 * pencil_tuned_cells);
    if (!need_sweep && !need_pencil) return NUC3D_OK;
    // NUC3D_SWEEP_RUN=1|2|4 pins the run length (32-cell tiles; with
    // NUC3D_SWEEP_TILE=64, runs of 2 or 4 on 64-cell tiles) and
    // NUC3D_PENCIL_DEPTH=16|32|64 the pencil depth (reproducibility studies)
    if (need_sweep) {
        if (const char *pin = std::getenv("NUC3D_SWEEP_RUN")) {
            const int run = std::atoi(pin);
            const char *tile = std::getenv("NUC3D_SWEEP_TILE");
            const int tc = tile && std::atoi(tile) == 64 && run != 1 && !mixed_tiles_only32()
                               ? 64
                               : 32;
            int v = 2;
            for (int k = 0; k < kInvVariants; ++k)
                if (kInvRunLen[k] == run && kInvTileCells[k] == tc) v = k;
            for (int s = 0; s < kSchemes; ++s)
                for (int d = 0; d < 3; ++d)
                    if (r_inv_[s][d][0].n > 0 && inv_variant[s][d] < 0) inv_variant[s][d] = v;
            need_sweep = false;
        }
    }
    bool tune_pencil = need_pencil;
    if (need_pencil) {
        if (const char *pin = std::getenv("NUC3D_PENCIL_DEPTH")) {
            const int want = std::atoi(pin);
            pencil_variant = 0;
            for (int v = 0; v < 3; ++v)
                if (kPencilDepths[v] == want) pencil_variant = v;
            pencil_tuned_cells = active_cells_;
            tune_pencil = false;
        }
    }
    invalidate_graph();
    if (!need_sweep && !tune_pencil) return NUC3D_OK;
    ECK(launch_prim(d_boxes_, d_items_ + r_prim_.off, r_prim_.n, 0, 0, stream_));
    cudaEvent_t e0, e1;
    ECK(cudaEventCreate(&e0));
    ECK(cudaEventCreate(&e1));
    const bool mixed = precision_ == NUC3D_MIXED;
    int rc = NUC3D_OK;
    // ms of one warm-up-then-3-repeats timing of go(), or a negative value
    // (with the error recorded) when a launch fails
    auto time3 = [&](auto &&go) -> double {
        cudaError_t err = go();  // warm-up
        err = err == cudaSuccess ? cudaEventRecord(e0, stream_) : err;
        for (int rep = 0; rep < 3 && err == cudaSuccess; ++rep) err = go();
        err = err == cudaSuccess ? cudaEventRecord(e1, stream_) : err;
        err = err == cudaSuccess ? cudaEventSynchronize(e1) : err;
        float ms = 0.f;
        err = err == cudaSuccess ? cudaEventElapsedTime(&ms, e0, e1) : err;
        if (err != cudaSuccess) {
            set_last_error(NUC3D_ERR_CUDA, cudaGetErrorString(err));
            rc = NUC3D_ERR_CUDA;
            return -1.0;
        }
        return ms / 3.0;
    };
    for (int s = 0; s < kSchemes && rc == NUC3D_OK && need_sweep; ++s)
        for (int d = 0; d < 3 && rc == NUC3D_OK; ++d) {
            if (r_inv_[s][d][0].n <= 0 || inv_variant[s][d] >= 0) continue;
            int best = 0;
            for (int v = 0; v < kInvVariants && rc == NUC3D_OK; ++v) {
                if (inv_tile_class(v) == 1 && mixed_tiles_only32()) {
                    inv_tune_ms[s][d][v] = 0.0;
                    continue;
                }
                const Range &rg = r_inv_[s][d][inv_tile_class(v)];
                // the x sweep is timed as the step runs it, recovering the
                // primitives of its tiles (prim_mode 1): it rewrites W with
                // bitwise the values k_prim has just written
                const int pm = d == 0 ? 1 : 0;
                const double ms = time3([&]() {
                    return mixed ? launch_inviscid<float>(s, d, v, d_boxes_, d_items_ + rg.off, rg.n,
                                                          0, d > 0, pm, stream_)
                                 : launch_inviscid<double>(s, d, v, d_boxes_, d_items_ + rg.off,
                                                           rg.n, 0, d > 0, pm, stream_);
                });
                inv_tune_ms[s][d][v] = ms;
                if (ms < inv_tune_ms[s][d][best]) best = v;
            }
            inv_variant[s][d] = best;
        }
    if (tune_pencil && rc == NUC3D_OK) {
        int best = 0;
        for (int v = 0; v < 3 && rc == NUC3D_OK; ++v) {
            const StageArgs sa{0, 0, 1, nullptr};
            const double ms = time3([&]() {
                cudaError_t err = cudaSuccess;
                if (any_visc_)
                    err = mixed ? launch_visc_classes<float>(v, stream_)
                                : launch_visc_classes<double>(v, stream_);
                if (err != cudaSuccess) return err;
                return mixed ? launch_update_classes<float>(v, sa, stream_)
                             : launch_update_classes<double>(v, sa, stream_);
            });
            pencil_tune_ms[v] = ms;
            if (ms < pencil_tune_ms[best]) best = v;
        }
        pencil_variant = best;
        pencil_tuned_cells = active_cells_;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    invalidate_graph();
    return rc;
}

int Engine::step(int nsteps) {
    if (nsteps < 0) return set_last_error(NUC3D_ERR_INVALID, "nsteps must be >= 0");
    if (dirty_) {
        int rc = rebuild();
        if (rc) return rc;
    }
    if (nactive_ == 0 || nsteps == 0) return NUC3D_OK;
    {
        int rc = autotune();
        if (rc) return rc;
    }
    if (prof_on) {
        for (int s = 0; s < nsteps; ++s) {
            int rc = enqueue_step(stream_);
            if (rc) return rc;
            launches += launches_per_step_;
            rc = profile_flush();
            if (rc) return rc;
        }
    } else {
        if (!exec_) {
            long long before = launches;
            if (!cap_stream_) ECK(cudaStreamCreateWithFlags(&cap_stream_, cudaStreamNonBlocking));
            if (!fork_stream_ && step_fork_enabled()) {
                ECK(cudaStreamCreateWithFlags(&fork_stream_, cudaStreamNonBlocking));
                for (cudaEvent_t &ev : fork_ev_)
                    ECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            }
            ECK(cudaStreamBeginCapture(cap_stream_, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue_step(cap_stream_);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(cap_stream_, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            ECK(e);
            graph_ = g;
            ECK(cudaGraphInstantiate(&exec_, graph_, 0));
            ++graph_captures;
            launches = before;
        }
        for (int s = 0; s < nsteps; ++s) ECK(cudaGraphLaunch(exec_, stream_));
        launches += (long long)nsteps * launches_per_step_;
    }
    for (auto &b : boxes_)
        if (b.live && b.dev.active) b.steps += nsteps;
    return NUC3D_OK;
}

int Engine::history(int id, int n, double *h_dt, double *h_res) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live)
        return set_last_error(NUC3D_ERR_INVALID, "no such box");
    if (n < 0 || n > kHistory) return set_last_error(NUC3D_ERR_INVALID, "history holds 1024 steps");
    const EngineBox &b = boxes_[id];
    if (n > b.steps) n = (int)b.steps;
    long long first = b.steps - n;
    int done = 0;
    while (done < n) {
        int ring = (int)((first + done) % kHistory);
        int cnt = std::min(n - done, kHistory - ring);
        if (h_dt)
            ECK(cudaMemcpyAsync(h_dt + done, b.dev.sc->dt_hist + ring, sizeof(double) * cnt,
                                cudaMemcpyDeviceToHost, stream_));
        if (h_res)
            ECK(cudaMemcpyAsync(h_res + done, b.dev.sc->res_hist + ring, sizeof(double) * cnt,
                                cudaMemcpyDeviceToHost, stream_));
        done += cnt;
    }
    ECK(cudaStreamSynchronize(stream_));
    return NUC3D_OK;
}

template <typename B>
int Engine::enqueue_rhs_t(int id, double *const d_rhs[5]) {
    const int nb = (int)boxes_.size();
    const WorkItem *it = d_items_;
    double *ptrs[5];
    for (int e = 0; e < 5; ++e) ptrs[e] = d_rhs[e];
    ECK(cudaMemcpyAsync(d_rhs_ptrs_ + 5 * id, ptrs, sizeof ptrs, cudaMemcpyHostToDevice, stream_));
    ECK(launch_clear_eig(d_boxes_, nb, stream_));
    ECK(launch_prim(d_boxes_, it + r_prim_.off, r_prim_.n, 0, 1, stream_));
    ECK(launch_dt(d_boxes_, nb, stream_));
    if (any_visc_) ECK(launch_visc_classes<B>(pv(), stream_));
    for (int d = 0; d < 3; ++d) {
        for (int s = 0; s < kSchemes; ++s)
            ECK((launch_inviscid<B>(s, d, inv_variant[s][d], d_boxes_, it + inv_range(s, d).off,
                                    inv_range(s, d).n, 0, d > 0, 0, stream_)));
        for (int c = 0; c < kLineSchemes; ++c)
            ECK((launch_crweno<B>(kLineScheme[c], d, d_boxes_, it + r_cr_[c][d].off,
                                  r_cr_[c][d].n, 0, d > 0, cr_nmax_[c][d], cr_ms_[c][d], 0,
                                  stream_)));
    }
    ECK(enqueue_forcing<B>(stream_));
    StageArgs sa{-1, 0, 0, d_rhs_ptrs_};
    ECK(launch_update_classes<B>(pv(), sa, stream_));
    ECK(cudaStreamSynchronize(stream_));  // ptrs is a host stack array
    return NUC3D_OK;
}

int Engine::rhs(int id, double *const d_rhs[5], double *h_dt_local) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live)
        return set_last_error(NUC3D_ERR_INVALID, "no such box");
    if (!d_rhs) return set_last_error(NUC3D_ERR_INVALID, "null argument");
    if (dirty_) {
        int rc = rebuild();
        if (rc) return rc;
    }
    if (nactive_ != 1 || !boxes_[id].dev.active)
        return set_last_error(NUC3D_ERR_UNSUPPORTED, "rhs needs exactly this one box active");
    {
        int rc = autotune();
        if (rc) return rc;
    }
    int rc = precision_ == NUC3D_MIXED ? enqueue_rhs_t<float>(id, d_rhs) : enqueue_rhs_t<double>(id, d_rhs);
    if (rc) return rc;
    if (h_dt_local) {
        ECK(cudaMemcpyAsync(h_dt_local, &boxes_[id].dev.sc->dt_local, sizeof(double),
                            cudaMemcpyDeviceToHost, stream_));
        ECK(cudaStreamSynchronize(stream_));
    }
    return NUC3D_OK;
}

int Engine::init_state(int id, const nuc3d_init_desc &in, double info[3]) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live)
        return set_last_error(NUC3D_ERR_INVALID, "no such box");
    EngineBox &b = boxes_[id];
    const BoxParams &p = b.dev.p;
    if (in.kind == NUC3D_INIT_TGV) {
        ECK(launch_init_tgv(b.dev, stream_));
        ECK(cudaStreamSynchronize(stream_));
        if (info) {
            info[0] = info[1] = NAN;
            info[2] = p.reynolds;
        }
        return NUC3D_OK;
    }
    if (in.kind != NUC3D_INIT_HIT) return set_last_error(NUC3D_ERR_INVALID, "unknown initial state kind");
    if (!(in.k_peak > 0.0) || !(in.mach_t > 0.0))
        return set_last_error(NUC3D_ERR_INVALID, "HIT needs k_peak > 0 and mach_t > 0");
    for (int d = 0; d < 3; ++d)
        if (hit_axis(p.n[d], 1.0, in.k_peak).M > 512)
            return set_last_error(NUC3D_ERR_INVALID, "HIT k_peak too large (at most 512 modes per axis)");
    // u_rms from the turbulent Mach number sqrt(3) u_rms / c with c = 1/M
    // (block.cpp:422 writes Mt / M^2 / sqrt(3): the same at M = 1)
    const double u_rms = in.mach_t / p.mach / std::sqrt(3.0);
    void *scratch = nullptr;
    double *d_sums = nullptr;
    const size_t bytes = hit_scratch_bytes(p, in.k_peak);
    cudaError_t e = cudaMallocAsync(&scratch, bytes + 256, stream_);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_last_error(NUC3D_ERR_NOMEM, "device allocation of the HIT scratch failed");
    }
    d_sums = reinterpret_cast<double *>(static_cast<char *>(scratch) + bytes);
    double sums[6] = {};
    e = launch_hit_synthesis(b.dev, b.desc.lx, b.desc.ly, b.desc.lz, in.seed, in.k_peak, u_rms,
                             scratch, d_sums, stream_);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sums, d_sums, sizeof sums, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    const double n = (double)p.N;
    const double cur = std::sqrt((sums[0] / n + sums[1] / n + sums[2] / n) / 3.0);
    const double scale = u_rms / cur;
    if (e == cudaSuccess) e = launch_hit_finalize(b.dev, scale, stream_);
    cudaError_t e2 = cudaFreeAsync(scratch, stream_);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    ECK(e);
    // Taylor microscale and Re_lambda as postproc.cpp:871-872 with rho = 1, T = 1
    const double u2 = (sums[0] / n + sums[1] / n + sums[2] / n) / 3.0 * scale * scale;
    const double d2 = (sums[3] / n + sums[4] / n + sums[5] / n) / 3.0 * scale * scale;
    const double lam = std::sqrt(u2 / d2), urms = std::sqrt(u2);
    if (in.re_lambda > 0.0) {
        const double re = in.re_lambda / (urms * lam);
        b.desc.reynolds = re;
        b.dev.p.reynolds = re;
        dirty_ = true;
    }
    if (info) {
        info[0] = urms;
        info[1] = lam;
        info[2] = b.dev.p.reynolds;
    }
    return NUC3D_OK;
}

int Engine::stats(int id, double out[26]) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live)
        return set_last_error(NUC3D_ERR_INVALID, "no such box");
    if (!out) return set_last_error(NUC3D_ERR_INVALID, "null argument");
    if (dirty_) {
        int rc = rebuild();
        if (rc) return rc;
    }
    EngineBox &b = boxes_[id];
    if (!b.dev.active) return set_last_error(NUC3D_ERR_INVALID, "box is not active");
    if (!d_stats_) ECK(cudaMallocAsync(&d_stats_, sizeof(double) * stats_scratch_doubles(), stream_));
    // primitives of U[0] into W (scratch between steps), then the sums
    ECK(launch_prim(d_boxes_, d_items_ + r_prim_.off + b.prim_off, b.prim_n, 0, 0, stream_));
    ECK(launch_stats(b.dev, d_stats_, stream_));
    double sums[kStatsSums];
    ECK(cudaMemcpyAsync(sums, d_stats_, sizeof sums, cudaMemcpyDeviceToHost, stream_));
    ECK(cudaStreamSynchronize(stream_));
    stats_finish(b.dev.p, sums, out);
    return NUC3D_OK;
}

int Engine::spectra(int id, double *out, int *kmax_out) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live)
        return set_last_error(NUC3D_ERR_INVALID, "no such box");
    if (!kmax_out) return set_last_error(NUC3D_ERR_INVALID, "null argument");
    if (dirty_) {
        int rc = rebuild();
        if (rc) return rc;
    }
    EngineBox &b = boxes_[id];
    const int kmax = spectra_kmax(b.dev.p);
    *kmax_out = kmax;
    if (!out) return NUC3D_OK;
    if (!b.dev.active) return set_last_error(NUC3D_ERR_INVALID, "box is not active");
    void *scratch = nullptr;
    double *d_out = nullptr;
    if (cudaMallocAsync(&scratch, spectra_scratch_bytes(b.dev.p), stream_) != cudaSuccess) {
        cudaGetLastError();
        return set_last_error(NUC3D_ERR_NOMEM, "no device memory for the spectra scratch");
    }
    int rc = NUC3D_OK;
    int fft_status = 0;
    cudaError_t e = cudaMallocAsync(&d_out, sizeof(double) * kSpectra * kmax, stream_);
    if (e == cudaSuccess)
        e = launch_prim(d_boxes_, d_items_ + r_prim_.off + b.prim_off, b.prim_n, 0, 0, stream_);
    if (e == cudaSuccess) e = launch_spectra(b.dev, scratch, d_out, &fft_status, stream_);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, d_out, sizeof(double) * kSpectra * kmax, cudaMemcpyDeviceToHost,
                            stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (fft_status != 0)
        rc = set_last_error(NUC3D_ERR_CUDA, ("cuFFT failed with status " +
                                             std::to_string(fft_status)).c_str());
    else if (e != cudaSuccess)
        rc = set_last_error(NUC3D_ERR_CUDA, cudaGetErrorString(e));
    cudaFreeAsync(scratch, stream_);
    if (d_out) cudaFreeAsync(d_out, stream_);
    return rc;
}

int Engine::sync_and_check(int id) {
    // The boxes' status flags reach the host through page-locked memory mapped
    // into the device, written by a one-warp kernel on this engine's stream:
    // no copy engine is involved, so the check cannot queue behind another
    // context's large state transfer (a synchronous cudaMemcpy of the flags
    // waited for such a transfer and released contexts in bursts).
    std::vector<int> ids;
    for (size_t i = 0; i < boxes_.size(); ++i)
        if (boxes_[i].live && (id < 0 || (int)i == id) && boxes_[i].dev.flags) ids.push_back((int)i);
    if ((int)ids.size() > h_flags_cap_) {
        if (h_flags_) cudaFreeHost(h_flags_);
        h_flags_ = nullptr;
        h_flags_cap_ = 0;
        const int cap = std::max(64, (int)ids.size());
        ECK(cudaHostAlloc(reinterpret_cast<void **>(&h_flags_), sizeof(unsigned) * cap,
                          cudaHostAllocMapped));
        h_flags_cap_ = cap;
        ECK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&h_flags_dev_), h_flags_, 0));
    }
    for (size_t c = 0; c < ids.size(); c += FlagPtrs::kMax) {
        FlagPtrs fp{};
        fp.n = (int)std::min(ids.size() - c, (size_t)FlagPtrs::kMax);
        for (int k = 0; k < fp.n; ++k) fp.p[k] = boxes_[ids[c + k]].dev.flags;
        k_export_flags<<<1, FlagPtrs::kMax, 0, stream_>>>(fp, h_flags_dev_ + c);
        ECK(cudaGetLastError());
    }
    ECK(cudaStreamSynchronize(stream_));
    for (size_t k = 0; k < ids.size(); ++k) {
        const unsigned f = reinterpret_cast<volatile unsigned *>(h_flags_)[k];
        if (f & kFlagWaitTimeout)
            return set_last_error(NUC3D_ERR_CUDA, "a bounded device wait timed out (viscous-flux TMA load)");
        if (f & kFlagNonFinite) return set_last_error(NUC3D_ERR_NONFINITE, "state became non-finite (NaN/Inf)");
    }
    return NUC3D_OK;
}

double Engine::time(int id) {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live) return NAN;
    double t = 0.0;
    if (cudaStreamSynchronize(stream_) != cudaSuccess) return NAN;
    if (cudaMemcpy(&t, &boxes_[id].dev.sc->time, sizeof t, cudaMemcpyDeviceToHost) != cudaSuccess)
        return NAN;
    return t;
}

long long Engine::box_steps(int id) const {
    if (id < 0 || id >= (int)boxes_.size() || !boxes_[id].live) return -1;
    return boxes_[id].steps;
}

}  // namespace nuc3d
