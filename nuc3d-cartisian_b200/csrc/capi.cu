// C ABI (include/nuc3d_b200.h): single-box contexts and batches (both thin
// handles over nuc3d::Engine), state transfer, the TVD-RK3 step driver and
// the per-operator entry points.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "engine.h"
#include "nuc3d_b200.h"
#include "nuc3d_device.cuh"
#include "op_kernels.h"
#include "rhs_kernels.h"

using namespace nuc3d;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char *where) {
    return fail(NUC3D_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
    } while (0)

}  // namespace

int nuc3d::set_last_error(int code, const char *msg) { return fail(code, msg); }

struct nuc3d_ctx {
    Engine *eng;
    int id;
};

struct nuc3d_batch {
    Engine *eng;
};

namespace {

// advance `nsteps`, reading dt/residual history per chunk of the device ring
int step_with_history(Engine *eng, int id, int nsteps, double *h_dt, double *h_res) {
    for (int s0 = 0; s0 < nsteps; s0 += kHistory) {
        int cnt = nsteps - s0 < kHistory ? nsteps - s0 : kHistory;
        int rc = eng->step(cnt);
        if (rc) return rc;
        if (h_dt || h_res) {
            rc = eng->history(id, cnt, h_dt ? h_dt + s0 : nullptr, h_res ? h_res + s0 : nullptr);
            if (rc) return rc;
        }
    }
    if (h_dt || h_res) return eng->sync_and_check(id);
    return NUC3D_OK;
}

int read_profile(Engine *eng, double *ms, long long *launches, int reset) {
    int rc = eng->profile_flush();
    if (rc) return rc;
    for (int i = 0; i < NUC3D_PROF_CLASSES; ++i) {
        if (ms) ms[i] = eng->prof_ms[i];
        if (launches) launches[i] = eng->prof_n[i];
        if (reset) {
            eng->prof_ms[i] = 0.0;
            eng->prof_n[i] = 0;
        }
    }
    return NUC3D_OK;
}

static_assert(kSchemes * 3 == NUC3D_TUNING_SLOTS, "tuning table layout");

// run lengths and times of the 32-cell-tile variants 0..2 (runs of 1, 2, 4)
int read_tuning(const Engine *eng, int *run_len, double *ms) {
    for (int s = 0; s < kSchemes; ++s)
        for (int d = 0; d < 3; ++d) {
            int v = eng->inv_variant[s][d];
            if (run_len) run_len[s * 3 + d] = v < 0 ? 0 : kInvRunLen[v];
            for (int k = 0; k < 3; ++k)
                if (ms) ms[(s * 3 + d) * 3 + k] = eng->inv_tune_ms[s][d][k];
        }
    return NUC3D_OK;
}

// tile lengths and times of the 64-cell-tile variants 3..4 (runs of 2, 4)
int read_tiles(const Engine *eng, int *tile_cells, double *ms64) {
    static_assert(kInvVariants == 5, "sweep tuning layout");
    for (int s = 0; s < kSchemes; ++s)
        for (int d = 0; d < 3; ++d) {
            int v = eng->inv_variant[s][d];
            if (tile_cells) tile_cells[s * 3 + d] = v < 0 ? 0 : kInvTileCells[v];
            for (int k = 0; k < 2; ++k)
                if (ms64) ms64[(s * 3 + d) * 2 + k] = eng->inv_tune_ms[s][d][3 + k];
        }
    return NUC3D_OK;
}

int read_pencil(const Engine *eng, int *depth, double *ms) {
    static_assert(NUC3D_PENCIL_DEPTHS == 3, "pencil tuning layout");
    if (depth) *depth = eng->pencil_variant < 0 ? 0 : kPencilDepths[eng->pencil_variant];
    for (int v = 0; v < 3; ++v)
        if (ms) ms[v] = eng->pencil_tune_ms[v];
    return NUC3D_OK;
}

}  // namespace

extern "C" {

int nuc3d_tuning_pencil(const nuc3d_ctx *c, int *depth, double *ms) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return read_pencil(c->eng, depth, ms);
}
int nuc3d_batch_tuning_pencil(const nuc3d_batch *b, int *depth, double *ms) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return read_pencil(b->eng, depth, ms);
}

int nuc3d_tuning_tiles(const nuc3d_ctx *c, int *tile_cells, double *ms64) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return read_tiles(c->eng, tile_cells, ms64);
}
int nuc3d_batch_tuning_tiles(const nuc3d_batch *b, int *tile_cells, double *ms64) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return read_tiles(b->eng, tile_cells, ms64);
}

int nuc3d_tuning(const nuc3d_ctx *c, int *run_len, double *ms) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return read_tuning(c->eng, run_len, ms);
}
int nuc3d_batch_tuning(const nuc3d_batch *b, int *run_len, double *ms) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return read_tuning(b->eng, run_len, ms);
}

const char *nuc3d_last_error(void) { return g_err.c_str(); }
const char *nuc3d_version(void) { return "nuc3d_b200 0.2 (sm_100a)"; }

void nuc3d_box_desc_default(nuc3d_box_desc *d) {
    if (!d) return;
    std::memset(d, 0, sizeof *d);
    d->nx = d->ny = d->nz = 64;
    d->lx = d->ly = d->lz = 2.0 * M_PI;
    d->scheme[0] = d->scheme[1] = d->scheme[2] = NUC3D_WENO5JS;
    d->pde_model = NUC3D_NAVIERSTOKES3D;
    d->visc_model = NUC3D_VISC_SUTHERLAND;
    d->gamma = 1.4;
    d->mach = 0.5;
    d->reynolds = 1000.0;
    d->prandtl = 0.72;
    d->t_ref = 110.4;
    d->t_inf = 288.0;
    d->powerlaw_exp = 0.76;
    d->precision = NUC3D_FP64;
    d->quirks = NUC3D_QUIRKS_REFERENCE;
    d->forcing = NUC3D_FORCING_NONE;
    d->forcing_amp = 0.01;  // physicsModel.cpp:37-39
    d->forcing_hel = 0.01;
    d->forcing_k = 1.0;
}

long long nuc3d_ctx_bytes(const nuc3d_box_desc *d) { return d ? Engine::box_bytes(*d) : -1; }

// ------------------------------------------------------------ contexts ----
int nuc3d_ctx_create(const nuc3d_box_desc *desc, void *stream, nuc3d_ctx **out) {
    if (!out) return fail(NUC3D_ERR_INVALID, "null output pointer");
    *out = nullptr;
    if (!desc) return fail(NUC3D_ERR_INVALID, "null box description");
    std::string why;
    int rc = Engine::validate(*desc, &why);
    if (rc) return fail(rc, why);
    Engine *eng = new (std::nothrow) Engine(desc->precision, static_cast<cudaStream_t>(stream));
    nuc3d_ctx *c = new (std::nothrow) nuc3d_ctx{eng, -1};
    if (!eng || !c) {
        delete eng;
        delete c;
        return fail(NUC3D_ERR_NOMEM, "host allocation failed");
    }
    rc = eng->add_box(*desc, &c->id);
    if (rc == NUC3D_OK) rc = eng->sync_and_check(c->id);
    if (rc) {
        delete eng;
        delete c;
        return rc;
    }
    *out = c;
    return NUC3D_OK;
}

int nuc3d_ctx_destroy(nuc3d_ctx *c) {
    if (!c) return NUC3D_OK;
    delete c->eng;
    delete c;
    return NUC3D_OK;
}

int nuc3d_set_state_host(nuc3d_ctx *c, const double *const h_q[5]) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return c->eng->set_state(c->id, h_q, cudaMemcpyHostToDevice, true);
}
int nuc3d_get_state_host(nuc3d_ctx *c, double *const h_q[5]) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return c->eng->get_state(c->id, h_q, cudaMemcpyDeviceToHost, true);
}
int nuc3d_set_state_host_async(nuc3d_ctx *c, const double *const h_q[5]) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return c->eng->set_state(c->id, h_q, cudaMemcpyHostToDevice, false);
}
int nuc3d_get_state_host_async(nuc3d_ctx *c, double *const h_q[5]) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return c->eng->get_state(c->id, h_q, cudaMemcpyDeviceToHost, false);
}
int nuc3d_ctx_copy_lane(nuc3d_ctx *c, int on) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    c->eng->copy_lane = on != 0;
    return NUC3D_OK;
}
int nuc3d_set_state_device(nuc3d_ctx *c, const double *const d_q[5]) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return c->eng->set_state(c->id, d_q, cudaMemcpyDeviceToDevice, false);
}
int nuc3d_get_state_device(nuc3d_ctx *c, double *const d_q[5]) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return c->eng->get_state(c->id, d_q, cudaMemcpyDeviceToDevice, false);
}

int nuc3d_step(nuc3d_ctx *c, int nsteps, double cfl, double *h_dt, double *h_res) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    if (nsteps < 0) return fail(NUC3D_ERR_INVALID, "nsteps must be >= 0");
    int rc = c->eng->set_cfl(c->id, cfl);
    if (rc) return rc;
    return step_with_history(c->eng, c->id, nsteps, h_dt, h_res);
}

int nuc3d_sync(nuc3d_ctx *c) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return c->eng->sync_and_check(c->id);
}

int nuc3d_rhs(nuc3d_ctx *c, double *const d_rhs[5], double *h_dt_local) {
    if (!c || !d_rhs) return fail(NUC3D_ERR_INVALID, "null argument");
    return c->eng->rhs(c->id, d_rhs, h_dt_local);
}

double nuc3d_ctx_time(const nuc3d_ctx *c) { return c ? c->eng->time(c->id) : NAN; }

int nuc3d_stats(nuc3d_ctx *c, double *h_out) {
    if (!c || !h_out) return fail(NUC3D_ERR_INVALID, "null argument");
    return c->eng->stats(c->id, h_out);
}
int nuc3d_spectra(nuc3d_ctx *c, double *h_out, int *kmax) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return c->eng->spectra(c->id, h_out, kmax);
}
int nuc3d_batch_spectra(nuc3d_batch *b, int box_id, double *h_out, int *kmax) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->spectra(box_id, h_out, kmax);
}
int nuc3d_batch_stats(nuc3d_batch *b, int box_id, double *h_out) {
    if (!b || !h_out) return fail(NUC3D_ERR_INVALID, "null argument");
    return b->eng->stats(box_id, h_out);
}

int nuc3d_init_state(nuc3d_ctx *c, const nuc3d_init_desc *init, double *h_info) {
    if (!c || !init) return fail(NUC3D_ERR_INVALID, "null argument");
    return c->eng->init_state(c->id, *init, h_info);
}

int nuc3d_profile_enable(nuc3d_ctx *c, int on) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    int rc = c->eng->profile_flush();
    c->eng->prof_on = on != 0;
    return rc;
}
int nuc3d_profile_read(nuc3d_ctx *c, double *ms, long long *launches, int reset) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return read_profile(c->eng, ms, launches, reset);
}
long long nuc3d_launch_count(const nuc3d_ctx *c) { return c ? c->eng->launches : 0; }

// -------------------------------------------------------------- batches ----
int nuc3d_batch_create(int precision, void *stream, nuc3d_batch **out) {
    if (!out) return fail(NUC3D_ERR_INVALID, "null output pointer");
    *out = nullptr;
    if (precision != NUC3D_FP64 && precision != NUC3D_MIXED)
        return fail(NUC3D_ERR_UNSUPPORTED, "unknown precision");
    Engine *eng = new (std::nothrow) Engine(precision, static_cast<cudaStream_t>(stream));
    nuc3d_batch *b = new (std::nothrow) nuc3d_batch{eng};
    if (!eng || !b) {
        delete eng;
        delete b;
        return fail(NUC3D_ERR_NOMEM, "host allocation failed");
    }
    *out = b;
    return NUC3D_OK;
}
int nuc3d_batch_destroy(nuc3d_batch *b) {
    if (!b) return NUC3D_OK;
    delete b->eng;
    delete b;
    return NUC3D_OK;
}
int nuc3d_batch_add(nuc3d_batch *b, const nuc3d_box_desc *d, int *box_id) {
    if (!b || !d || !box_id) return fail(NUC3D_ERR_INVALID, "null argument");
    return b->eng->add_box(*d, box_id);
}
int nuc3d_batch_remove(nuc3d_batch *b, int box_id) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->remove_box(box_id);
}
int nuc3d_batch_set_active(nuc3d_batch *b, int box_id, int active) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->set_active(box_id, active != 0);
}
int nuc3d_batch_set_cfl(nuc3d_batch *b, int box_id, double cfl) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->set_cfl(box_id, cfl);
}
int nuc3d_batch_init_state(nuc3d_batch *b, int box_id, const nuc3d_init_desc *init,
                           double *h_info) {
    if (!b || !init) return fail(NUC3D_ERR_INVALID, "null argument");
    return b->eng->init_state(box_id, *init, h_info);
}
int nuc3d_batch_set_state_host(nuc3d_batch *b, int box_id, const double *const h_q[5]) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->set_state(box_id, h_q, cudaMemcpyHostToDevice, true);
}
int nuc3d_batch_get_state_host(nuc3d_batch *b, int box_id, double *const h_q[5]) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->get_state(box_id, h_q, cudaMemcpyDeviceToHost, true);
}
int nuc3d_batch_set_state_device(nuc3d_batch *b, int box_id, const double *const d_q[5]) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->set_state(box_id, d_q, cudaMemcpyDeviceToDevice, false);
}
int nuc3d_batch_get_state_device(nuc3d_batch *b, int box_id, double *const d_q[5]) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->get_state(box_id, d_q, cudaMemcpyDeviceToDevice, false);
}
int nuc3d_batch_step(nuc3d_batch *b, int nsteps) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->step(nsteps);
}
int nuc3d_batch_history(nuc3d_batch *b, int box_id, int n, double *h_dt, double *h_res) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->history(box_id, n, h_dt, h_res);
}
int nuc3d_batch_sync(nuc3d_batch *b) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return b->eng->sync_and_check(-1);
}
long long nuc3d_batch_box_steps(const nuc3d_batch *b, int box_id) {
    return b ? b->eng->box_steps(box_id) : -1;
}
double nuc3d_batch_time(nuc3d_batch *b, int box_id) { return b ? b->eng->time(box_id) : NAN; }
int nuc3d_batch_profile_enable(nuc3d_batch *b, int on) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    int rc = b->eng->profile_flush();
    b->eng->prof_on = on != 0;
    return rc;
}
int nuc3d_batch_profile_read(nuc3d_batch *b, double *ms, long long *launches, int reset) {
    if (!b) return fail(NUC3D_ERR_INVALID, "null batch");
    return read_profile(b->eng, ms, launches, reset);
}
long long nuc3d_batch_launch_count(const nuc3d_batch *b) { return b ? b->eng->launches : 0; }

// -------------------------------------------------------- per-operator ----
int nuc3d_reconstruct(int scheme, int upwind, unsigned quirks, int nx, int ny, int nz,
                      const double *in, const double *hl, const double *hr, double *out,
                      void *stream) {
    if (scheme < NUC3D_WENO5JS || scheme > NUC3D_UPWIND1ST)
        return fail(NUC3D_ERR_UNSUPPORTED, "weno error: no such scheme");
    if (upwind != 1 && upwind != -1) return fail(NUC3D_ERR_INVALID, "weno error: no such direction");
    if (nx < 8 || ny < 1 || nz < 1) return fail(NUC3D_ERR_INVALID, "need nx >= 8, ny, nz >= 1");
    if ((scheme == NUC3D_CRWENO5 || scheme == NUC3D_HCCS || scheme == NUC3D_HCCS77) && nx > 4096)
        return fail(NUC3D_ERR_INVALID, "crweno5 / hccs / hccs77 need nx <= 4096");
    if ((scheme == NUC3D_HCCS || scheme == NUC3D_HCCS77) && nx < 9)
        return fail(NUC3D_ERR_INVALID, "hccs / hccs77 need nx >= 9");
    if (!in || !hl || !hr || !out) return fail(NUC3D_ERR_INVALID, "null buffer");
    CK(op_reconstruct(scheme, upwind, quirks, nx, (long long)ny * nz, in, hl, hr, out,
                      static_cast<cudaStream_t>(stream)));
    return NUC3D_OK;
}

int nuc3d_cd6(int nx, int ny, int nz, double dx, const double *in, const double *hl,
              const double *hr, double *out, void *stream) {
    if (nx < 6 || ny < 1 || nz < 1 || !(dx > 0.0)) return fail(NUC3D_ERR_INVALID, "bad size or dx");
    if (!in || !hl || !hr || !out) return fail(NUC3D_ERR_INVALID, "null buffer");
    CK(op_cd6(nx, (long long)ny * nz, dx, in, hl, hr, out, static_cast<cudaStream_t>(stream)));
    return NUC3D_OK;
}

int nuc3d_differential(int scheme, int tile, int nx, int ny, int nz, double dx, const double *in,
                       const double *hl, const double *hr, double *out, void *stream) {
    if (scheme < NUC3D_CD6 || scheme > NUC3D_CD8) return fail(NUC3D_ERR_UNSUPPORTED, "unknown differential scheme");
    const int reach = scheme == NUC3D_CD2 ? 1 : (scheme == NUC3D_CD8 ? 4 : 3);
    if (tile < reach || tile > 4)
        return fail(NUC3D_ERR_INVALID, "tilesize must cover the stencil's reach and be <= 4");
    if (nx < 2 * tile || nx > 4096 || ny < 1 || nz < 1 || !(dx > 0.0))
        return fail(NUC3D_ERR_INVALID, "bad size or dx");
    if (!in || !hl || !hr || !out) return fail(NUC3D_ERR_INVALID, "null buffer");
    CK(op_differential(scheme, tile, nx, (long long)ny * nz, dx, in, hl, hr, out,
                       static_cast<cudaStream_t>(stream)));
    return NUC3D_OK;
}

int nuc3d_tvdrk3_stage(int stage, long long n, double dt, const double *const d_rhs[5],
                       const double *const d_un[5], double *const d_ui[5], void *stream) {
    if (stage < 0 || stage > 2) return fail(NUC3D_ERR_INVALID, "stage must be 0, 1 or 2");
    if (n < 0 || !d_rhs || !d_un || !d_ui) return fail(NUC3D_ERR_INVALID, "bad argument");
    RK5 rk;
    for (int e = 0; e < 5; ++e) {
        rk.rhs[e] = d_rhs[e];
        rk.un[e] = d_un[e];
        rk.ui[e] = d_ui[e];
    }
    if (n == 0) return NUC3D_OK;
    CK(op_rk3(stage, n, dt, rk, static_cast<cudaStream_t>(stream)));
    return NUC3D_OK;
}

}  // extern "C"
