// C ABI (include/nuc3d_b200.h): contexts, state transfer, the TVD-RK3 step
// driver and the per-operator entry points.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

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

long long pad32(long long n) { return (n + 31) / 32 * 32; }

int validate(const nuc3d_box_desc *d) {
    if (!d) return fail(NUC3D_ERR_INVALID, "null box description");
    const int n[3] = {d->nx, d->ny, d->nz};
    for (int i = 0; i < 3; ++i) {
        if (n[i] < 8) return fail(NUC3D_ERR_INVALID, "every box extent must be >= 8 cells");
        if (d->scheme[i] < NUC3D_WENO5JS || d->scheme[i] > NUC3D_CRWENO5)
            return fail(NUC3D_ERR_UNSUPPORTED, "unknown reconstruction scheme");
    }
    if ((long long)d->nx * d->ny * d->nz > (1LL << 31))
        return fail(NUC3D_ERR_INVALID, "box larger than 2^31 cells");
    if (!(d->lx > 0 && d->ly > 0 && d->lz > 0)) return fail(NUC3D_ERR_INVALID, "box lengths must be > 0");
    if (d->pde_model != NUC3D_EULER3D && d->pde_model != NUC3D_NAVIERSTOKES3D)
        return fail(NUC3D_ERR_UNSUPPORTED, "unknown PDE model");
    if (d->visc_model < NUC3D_VISC_SUTHERLAND || d->visc_model > NUC3D_VISC_POWERLAW)
        return fail(NUC3D_ERR_UNSUPPORTED, "unknown viscosity model");
    if (d->precision != NUC3D_FP64 && d->precision != NUC3D_MIXED)
        return fail(NUC3D_ERR_UNSUPPORTED, "unknown precision");
    if (!(d->gamma > 1.0) || !(d->mach > 0.0) || !(d->reynolds > 0.0) || !(d->prandtl > 0.0))
        return fail(NUC3D_ERR_INVALID, "gamma must be > 1 and Mach, Re, Pr > 0");
    return NUC3D_OK;
}

}  // namespace

int nuc3d::set_last_error(int code, const char *msg) { return fail(code, msg); }

struct nuc3d_ctx {
    nuc3d_box_desc desc;
    BoxParams bp;
    cudaStream_t stream;
    int sms;
    long long npad;
    void *mem_dp;    // FP64 fields: U[3][5], W[6]
    void *mem_bulk;  // bulk fields: R[5], V[9]
    void *mem_scratch;
    void *mem_small;  // eig[4], res_acc, flags, StepScalars
    double *U[3][5];
    double *W[6];
    void *R[5];
    void *V[9];
    double *eig;
    double *res_acc;
    unsigned *flags;
    StepScalars *sc;
    double time_host;
    // kernel accounting
    long long launches = 0;
    bool prof_on = false;
    std::vector<cudaEvent_t> ev_pool;
    struct Mark {
        int cls;
        cudaEvent_t a, b;
    };
    std::vector<Mark> pending;
    size_t ev_next = 0;
    double prof_ms[NUC3D_PROF_CLASSES] = {};
    long long prof_n[NUC3D_PROF_CLASSES] = {};
};

namespace {

size_t bulk_size(const nuc3d_box_desc *d) {
    return d->precision == NUC3D_MIXED ? sizeof(float) : sizeof(double);
}
bool any_crweno(const nuc3d_box_desc *d) {
    return d->scheme[0] == NUC3D_CRWENO5 || d->scheme[1] == NUC3D_CRWENO5 ||
           d->scheme[2] == NUC3D_CRWENO5;
}
BoxParams make_params(const nuc3d_box_desc *d) {
    BoxParams bp{};
    bp.n[0] = d->nx;
    bp.n[1] = d->ny;
    bp.n[2] = d->nz;
    bp.N = (long long)d->nx * d->ny * d->nz;
    bp.stride[0] = 1;
    bp.stride[1] = d->nx;
    bp.stride[2] = (long long)d->nx * d->ny;
    bp.d[0] = d->lx / d->nx;  // block.cpp:62-64
    bp.d[1] = d->ly / d->ny;
    bp.d[2] = d->lz / d->nz;
    for (int i = 0; i < 3; ++i) bp.inv_d[i] = 1.0 / bp.d[i];
    bp.gamma = d->gamma;
    bp.mach = d->mach;
    bp.reynolds = d->reynolds;
    bp.prandtl = d->prandtl;
    bp.tref_nd = d->t_ref / d->t_inf;
    bp.powerlaw_exp = d->powerlaw_exp;
    bp.cfl = 0.5;
    bp.visc_model = d->visc_model;
    bp.navier_stokes = d->pde_model == NUC3D_NAVIERSTOKES3D;
    bp.quirks = d->quirks;
    for (int i = 0; i < 3; ++i) bp.scheme[i] = d->scheme[i];
    return bp;
}
size_t small_bytes() { return 256 + sizeof(StepScalars); }

// Event bracketing of one launch (or a run of launches of one class).
cudaEvent_t pool_event(nuc3d_ctx *c) {
    if (c->ev_next == c->ev_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[c->ev_next++];
}
struct ProfScope {
    nuc3d_ctx *c;
    int cls;
    cudaEvent_t a = nullptr;
    ProfScope(nuc3d_ctx *c_, int cls_) : c(c_), cls(cls_) {
        if (c->prof_on && (a = pool_event(c))) cudaEventRecord(a, c->stream);
    }
    ~ProfScope() {
        if (!a) return;
        cudaEvent_t b = pool_event(c);
        if (!b) return;
        cudaEventRecord(b, c->stream);
        c->pending.push_back({cls, a, b});
    }
};
int prof_flush(nuc3d_ctx *c) {
    if (c->pending.empty()) return NUC3D_OK;
    CK(cudaStreamSynchronize(c->stream));
    for (auto &m : c->pending) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, m.a, m.b));
        c->prof_ms[m.cls] += ms;
        c->prof_n[m.cls] += 1;
    }
    c->pending.clear();
    c->ev_next = 0;
    return NUC3D_OK;
}

// one RHS evaluation of state `in` into R (and V); stage >= 0 selects RK
template <typename B>
int rhs_into_r(nuc3d_ctx *c, double *const in[5], int want_eig, int step) {
    const BoxParams &bp = c->bp;
    StateView q{{in[0], in[1], in[2], in[3], in[4]}};
    PrimView w{{c->W[0], c->W[1], c->W[2], c->W[3], c->W[4], c->W[5]}};
    BView<B> r;
    for (int e = 0; e < 5; ++e) r.f[e] = static_cast<B *>(c->R[e]);
    BView9<B> vf;
    for (int e = 0; e < 9; ++e) vf.f[e] = static_cast<B *>(c->V[e]);
    {
        ProfScope ps(c, NUC3D_PROF_PRIM);
        CK(launch_prim(bp, q, w, c->eig, want_eig, c->sms, c->stream));
        ++c->launches;
    }
    if (want_eig) {
        ProfScope ps(c, NUC3D_PROF_DT);
        CK(launch_dt(bp, c->eig, c->sc, step, c->stream));
        ++c->launches;
    }
    if (bp.navier_stokes) {
        ProfScope ps(c, NUC3D_PROF_VISC);
        CK((launch_visc_flux<B>(bp, w, vf, c->sms, c->stream)));
        ++c->launches;
    }
    for (int d = 0; d < 3; ++d) {
        ProfScope ps(c, NUC3D_PROF_INV_X + d);
        if (bp.scheme[d] == SCHEME_CR) {
            int nl = 0;
            CK((launch_crweno<B>(bp, d, q, w, r, d > 0, static_cast<B *>(c->mem_scratch), c->stream,
                                 &nl)));
            c->launches += nl;
        } else {
            CK((launch_inviscid<B>(bp, d, q, w, r, d > 0, c->stream)));
            ++c->launches;
        }
    }
    return NUC3D_OK;
}

template <typename B>
int update(nuc3d_ctx *c, double *const in[5], double *const out[5], int stage) {
    BView<B> r;
    for (int e = 0; e < 5; ++e) r.f[e] = static_cast<B *>(c->R[e]);
    BView9<B> vf;
    for (int e = 0; e < 9; ++e) vf.f[e] = static_cast<B *>(c->V[e]);
    StateView un{{c->U[0][0], c->U[0][1], c->U[0][2], c->U[0][3], c->U[0][4]}};
    StateView ui{{in[0], in[1], in[2], in[3], in[4]}};
    StateViewMut uo{{out[0], out[1], out[2], out[3], out[4]}};
    ProfScope ps(c, NUC3D_PROF_UPDATE);
    CK((launch_update<B>(c->bp, r, vf, un, ui, uo, stage, c->sc, c->res_acc, c->flags, c->sms,
                         c->stream)));
    ++c->launches;
    return NUC3D_OK;
}

template <typename B>
int one_step(nuc3d_ctx *c, int hist_slot) {
    CK(cudaMemsetAsync(c->eig, 0, 4 * sizeof(double), c->stream));
    for (int stage = 0; stage < 3; ++stage) {
        double *const *in = c->U[stage];            // u_n, u1, u2
        double *const *out = c->U[(stage + 1) % 3];  // u1, u2, u_n (in place)
        int rc = rhs_into_r<B>(c, in, stage == 0, hist_slot);
        if (rc) return rc;
        rc = update<B>(c, in, out, stage);
        if (rc) return rc;
    }
    {
        ProfScope ps(c, NUC3D_PROF_RESIDUAL);
        CK(launch_residual(c->bp, c->sc, c->res_acc, hist_slot, c->stream));
        ++c->launches;
    }
    return c->prof_on ? prof_flush(c) : NUC3D_OK;
}

int check_flags(nuc3d_ctx *c) {
    unsigned f = 0;
    CK(cudaMemcpyAsync(&f, c->flags, sizeof f, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (f & 1u) return fail(NUC3D_ERR_NONFINITE, "state became non-finite (NaN/Inf)");
    return NUC3D_OK;
}

}  // namespace

extern "C" {

const char *nuc3d_last_error(void) { return g_err.c_str(); }
const char *nuc3d_version(void) { return "nuc3d_b200 0.1 (sm_100a)"; }

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
}

long long nuc3d_ctx_bytes(const nuc3d_box_desc *d) {
    if (validate(d) != NUC3D_OK) return -1;
    BoxParams bp = make_params(d);
    long long np = pad32(bp.N);
    long long b = 21 * np * 8 + 14 * np * (long long)bulk_size(d) + (long long)small_bytes();
    if (any_crweno(d)) b += (long long)crweno_scratch_elems(bp) * (long long)bulk_size(d);
    return b;
}

int nuc3d_ctx_create(const nuc3d_box_desc *desc, void *stream, nuc3d_ctx **out) {
    if (!out) return fail(NUC3D_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int rc = validate(desc);
    if (rc) return rc;
    nuc3d_ctx *c = new (std::nothrow) nuc3d_ctx();
    if (!c) return fail(NUC3D_ERR_NOMEM, "host allocation failed");
    c->desc = *desc;
    c->bp = make_params(desc);
    c->stream = static_cast<cudaStream_t>(stream);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(e, "cudaGetDevice");
    }
    c->npad = pad32(c->bp.N);
    size_t bs = bulk_size(desc);
    size_t dp_bytes = sizeof(double) * 21 * (size_t)c->npad;
    size_t bulk_bytes = bs * 14 * (size_t)c->npad;
    size_t scr_bytes = any_crweno(desc) ? bs * crweno_scratch_elems(c->bp) : 0;
    e = cudaMalloc(&c->mem_dp, dp_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&c->mem_bulk, bulk_bytes);
    if (e == cudaSuccess && scr_bytes) e = cudaMalloc(&c->mem_scratch, scr_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&c->mem_small, small_bytes());
    if (e != cudaSuccess) {
        cudaFree(c->mem_dp);
        cudaFree(c->mem_bulk);
        cudaFree(c->mem_scratch);
        cudaFree(c->mem_small);
        delete c;
        cudaGetLastError();
        return fail(NUC3D_ERR_NOMEM, std::string("device allocation failed: ") + cudaGetErrorString(e));
    }
    double *dp = static_cast<double *>(c->mem_dp);
    for (int s = 0; s < 3; ++s)
        for (int q = 0; q < 5; ++q) c->U[s][q] = dp + (size_t)(s * 5 + q) * c->npad;
    for (int i = 0; i < 6; ++i) c->W[i] = dp + (size_t)(15 + i) * c->npad;
    char *bk = static_cast<char *>(c->mem_bulk);
    for (int i = 0; i < 5; ++i) c->R[i] = bk + bs * (size_t)i * c->npad;
    for (int i = 0; i < 9; ++i) c->V[i] = bk + bs * (size_t)(5 + i) * c->npad;
    char *sm = static_cast<char *>(c->mem_small);
    c->eig = reinterpret_cast<double *>(sm);
    c->res_acc = reinterpret_cast<double *>(sm + 64);
    c->flags = reinterpret_cast<unsigned *>(sm + 128);
    c->sc = reinterpret_cast<StepScalars *>(sm + 256);
    e = cudaMemsetAsync(c->mem_small, 0, small_bytes(), c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->mem_dp, 0, dp_bytes, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->mem_bulk, 0, bulk_bytes, c->stream);
    if (e != cudaSuccess) {
        nuc3d_ctx_destroy(c);
        return cuda_fail(e, "cudaMemsetAsync");
    }
    *out = c;
    return NUC3D_OK;
}

int nuc3d_ctx_destroy(nuc3d_ctx *c) {
    if (!c) return NUC3D_OK;
    cudaStreamSynchronize(c->stream);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    cudaFree(c->mem_dp);
    cudaFree(c->mem_bulk);
    cudaFree(c->mem_scratch);
    cudaFree(c->mem_small);
    delete c;
    return NUC3D_OK;
}

static int copy_state(nuc3d_ctx *c, double *const dst[5], const double *const src[5],
                      cudaMemcpyKind kind, bool sync) {
    if (!c || !dst || !src) return fail(NUC3D_ERR_INVALID, "null argument");
    size_t bytes = sizeof(double) * (size_t)c->bp.N;
    for (int e = 0; e < 5; ++e) {
        if (!dst[e] || !src[e]) return fail(NUC3D_ERR_INVALID, "null field pointer");
        CK(cudaMemcpyAsync(dst[e], src[e], bytes, kind, c->stream));
    }
    if (sync) CK(cudaStreamSynchronize(c->stream));
    return NUC3D_OK;
}

int nuc3d_set_state_host(nuc3d_ctx *c, const double *const h_q[5]) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return copy_state(c, c->U[0], h_q, cudaMemcpyHostToDevice, true);
}
int nuc3d_get_state_host(nuc3d_ctx *c, double *const h_q[5]) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return copy_state(c, h_q, c->U[0], cudaMemcpyDeviceToHost, true);
}
int nuc3d_set_state_device(nuc3d_ctx *c, const double *const d_q[5]) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return copy_state(c, c->U[0], d_q, cudaMemcpyDeviceToDevice, false);
}
int nuc3d_get_state_device(nuc3d_ctx *c, double *const d_q[5]) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return copy_state(c, d_q, c->U[0], cudaMemcpyDeviceToDevice, false);
}

int nuc3d_step(nuc3d_ctx *c, int nsteps, double cfl, double *h_dt, double *h_res) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    if (nsteps < 0) return fail(NUC3D_ERR_INVALID, "nsteps must be >= 0");
    if (!(cfl > 0.0)) return fail(NUC3D_ERR_INVALID, "cfl must be > 0");
    c->bp.cfl = cfl;
    const bool mixed = c->desc.precision == NUC3D_MIXED;
    for (int s0 = 0; s0 < nsteps; s0 += kHistory) {
        int cnt = nsteps - s0 < kHistory ? nsteps - s0 : kHistory;
        for (int s = 0; s < cnt; ++s) {
            int rc = mixed ? one_step<float>(c, s) : one_step<double>(c, s);
            if (rc) return rc;
        }
        if (h_dt)
            CK(cudaMemcpyAsync(h_dt + s0, c->sc->dt_hist, sizeof(double) * cnt,
                               cudaMemcpyDeviceToHost, c->stream));
        if (h_res)
            CK(cudaMemcpyAsync(h_res + s0, c->sc->res_hist, sizeof(double) * cnt,
                               cudaMemcpyDeviceToHost, c->stream));
    }
    if (h_dt || h_res) return check_flags(c);
    return NUC3D_OK;
}

int nuc3d_sync(nuc3d_ctx *c) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    return check_flags(c);
}

int nuc3d_rhs(nuc3d_ctx *c, double *const d_rhs[5], double *h_dt_local) {
    if (!c || !d_rhs) return fail(NUC3D_ERR_INVALID, "null argument");
    CK(cudaMemsetAsync(c->eig, 0, 4 * sizeof(double), c->stream));
    const bool mixed = c->desc.precision == NUC3D_MIXED;
    int rc = mixed ? rhs_into_r<float>(c, c->U[0], 1, -1) : rhs_into_r<double>(c, c->U[0], 1, -1);
    if (rc) return rc;
    rc = mixed ? update<float>(c, c->U[0], d_rhs, -1) : update<double>(c, c->U[0], d_rhs, -1);
    if (rc) return rc;
    if (h_dt_local) {
        CK(cudaMemcpyAsync(h_dt_local, &c->sc->dt_local, sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return NUC3D_OK;
}

int nuc3d_profile_enable(nuc3d_ctx *c, int on) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    int rc = prof_flush(c);
    c->prof_on = on != 0;
    return rc;
}

int nuc3d_profile_read(nuc3d_ctx *c, double *ms, long long *launches, int reset) {
    if (!c) return fail(NUC3D_ERR_INVALID, "null context");
    int rc = prof_flush(c);
    if (rc) return rc;
    for (int i = 0; i < NUC3D_PROF_CLASSES; ++i) {
        if (ms) ms[i] = c->prof_ms[i];
        if (launches) launches[i] = c->prof_n[i];
        if (reset) {
            c->prof_ms[i] = 0.0;
            c->prof_n[i] = 0;
        }
    }
    return NUC3D_OK;
}

long long nuc3d_launch_count(const nuc3d_ctx *c) { return c ? c->launches : 0; }

double nuc3d_ctx_time(const nuc3d_ctx *c) {
    if (!c) return 0.0;
    double t = 0.0;
    if (cudaMemcpy(&t, &c->sc->time, sizeof t, cudaMemcpyDeviceToHost) != cudaSuccess) return NAN;
    return t;
}

int nuc3d_reconstruct(int scheme, int upwind, unsigned quirks, int nx, int ny, int nz,
                      const double *in, const double *hl, const double *hr, double *out,
                      void *stream) {
    if (scheme < NUC3D_WENO5JS || scheme > NUC3D_CRWENO5)
        return fail(NUC3D_ERR_UNSUPPORTED, "weno error: no such scheme");
    if (upwind != 1 && upwind != -1) return fail(NUC3D_ERR_INVALID, "weno error: no such direction");
    if (nx < 8 || ny < 1 || nz < 1) return fail(NUC3D_ERR_INVALID, "need nx >= 8, ny, nz >= 1");
    if (scheme == NUC3D_CRWENO5 && nx > 4096) return fail(NUC3D_ERR_INVALID, "crweno5 needs nx <= 4096");
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
