/*
 * nuc3d_b200 — C ABI of the B200-native NUC3d RHS + TVD-RK3 path.
 *
 * Plain C types only (pointers, sizes, doubles); no CUDA or torch types.  A
 * stream is passed as `void *` holding a cudaStream_t (NULL = legacy default
 * stream).  Every entry point returns an int status (NUC3D_OK = 0, negative on
 * error) and never aborts the process: the reference's error behaviour
 * (print + exit(-1) / MPI_Abort, e.g. weno5js.cpp:32-34) becomes a status code
 * plus nuc3d_last_error() text.
 *
 * Fields are FP64, x-fastest, idx = i + nx*(j + ny*k): the layout of the
 * reference's Field (field.h:9-79, block.cpp:119).  Device pointers are
 * marked d_*, host pointers h_*.
 */
#ifndef NUC3D_B200_H
#define NUC3D_B200_H

#if defined(__GNUC__)
#define NUC3D_API __attribute__((visibility("default")))
#else
#define NUC3D_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define NUC3D_OK 0
#define NUC3D_ERR_INVALID (-1)     /* bad argument or size */
#define NUC3D_ERR_CUDA (-2)        /* a CUDA call failed */
#define NUC3D_ERR_NOMEM (-3)       /* device allocation failed */
#define NUC3D_ERR_UNSUPPORTED (-4) /* scheme / model not available */
#define NUC3D_ERR_NONFINITE (-5)   /* the state went NaN/Inf (finite check) */
#define NUC3D_ERR_TIMEOUT (-6)     /* nuc3d_serve_wait: not finished in time */
#define NUC3D_ERR_CANCELLED (-7)   /* solve dropped by nuc3d_serve_destroy */

/* Reconstruction schemes: the Method.in strings weno5js, weno5z, crweno5,
 * weno7js, hccs, hccs77, hccs78, weno3js, upwind1st (fieldOperator.cpp:
 * 128-189).  weno7js and the hccs family read 4 halo cells per side (their
 * bufferSize), weno3js 2, upwind1st 1, the others 3.  hccs is the hybrid compact scheme of hccs.cpp (WENO7 end faces,
 * linear upwind compact rows blended with CRWENO5-weighted rows); hccs77
 * (hccs77.cpp) blends WENO7-Z into the 7th-order upwind compact rows; their
 * lines are bounded tridiagonal systems like crweno5's reference form.
 * hccs78 (hccs78.cpp) is explicit: WENO7-Z blended with the 8th-order
 * central value on the inner faces, WENO7-Z at the ends. */
#define NUC3D_WENO5JS 0
#define NUC3D_WENO5Z 1
#define NUC3D_CRWENO5 2
#define NUC3D_WENO7JS 3
#define NUC3D_HCCS 4
#define NUC3D_HCCS77 5
#define NUC3D_HCCS78 6
#define NUC3D_WENO3JS 7
#define NUC3D_UPWIND1ST 8

/* PDEModel (block.cpp:146-157) */
#define NUC3D_EULER3D 0
#define NUC3D_NAVIERSTOKES3D 1

/* ViscousModel (physicsModel.cpp:44-49); POWERLAW mu = T^w / Re is an extra
 * model the reference does not have. */
#define NUC3D_VISC_SUTHERLAND 0
#define NUC3D_VISC_CONSTANT 1
#define NUC3D_VISC_POWERLAW 2

/* Arithmetic of the bulk (reconstruction, flux differences, viscous
 * stencils).  The conserved state, pressure/temperature recovery, the RK
 * accumulation and all global reductions are FP64 in both. */
#define NUC3D_FP64 0
#define NUC3D_MIXED 1

/* Reference behaviours that look like defects.  Each is reproduced while its
 * bit is set; NUC3D_QUIRKS_REFERENCE (all set) is the drop-in default. */
#define NUC3D_QUIRK_ZETA_EIGEN 0x1u     /* physicsModel.cpp:653-654, euler3d.cpp:459-466 */
#define NUC3D_QUIRK_WENOZ_BETA2 0x2u    /* weno5z.cpp:80 */
#define NUC3D_QUIRK_OFFDIAG_DIV 0x4u    /* NaiverStokes3d.cpp:267-270 */
#define NUC3D_QUIRK_FABS_PRESSURE 0x8u  /* physicsModel.cpp:340 */
#define NUC3D_QUIRK_CRWENO_BOUNDED 0x10u /* crweno5.cpp:45-402 (cleared: periodic lines) */
#define NUC3D_QUIRKS_REFERENCE 0x1fu

typedef struct nuc3d_box_desc {
    int nx, ny, nz;          /* cells; block.in line 2 (single rank) */
    double lx, ly, lz;       /* box lengths; dx = lx/nx (block.cpp:62-64) */
    int scheme[3];           /* scheme_{x,y,z}_ivs */
    int pde_model;           /* PDEModel */
    int visc_model;          /* ViscousModel */
    double gamma, mach, reynolds, prandtl, t_ref, t_inf; /* PhysModel.in keys */
    double powerlaw_exp;     /* exponent of NUC3D_VISC_POWERLAW */
    int precision;           /* NUC3D_FP64 or NUC3D_MIXED */
    unsigned quirks;         /* NUC3D_QUIRK_* mask */
    /* PhysModel.in Forcing (physicsModel.cpp:50-56): NUC3D_FORCING_NONE or
     * NUC3D_FORCING_CONST, the spectral shell forcing of AddForcing_Const
     * (physicsModel.cpp:1368-1641) with Forcing_amplitude (target shell
     * energy), Forcing_amplitude_hel (helical part) and Forcing_wave_k (shell
     * radius, < 3.5).
     * NUC3D_FORCING_BAND (no counterpart in the reference, which has only
     * the shell forcing): band-limited forcing at a fixed energy-injection
     * rate.  On every RHS evaluation the solenoidal part s(k) of the
     * velocity's Fourier modes with 0 < |k| <= forcing_k (< 3.5) is forced
     * as f(k) = P s(k) / (2 E_b), E_b = sum over the band of |s(k)|^2 / 2,
     * P = forcing_amp, so that the mean kinetic-energy input <f.u> is
     * exactly P; forcing_hel is ignored.  It enters the RHS as the shell
     * forcing does (density taken as 1; energy equation gets f.u - <f.u>). */
    int forcing;
    double forcing_amp, forcing_hel, forcing_k;
    /* PhysModel.in RiemannSolver (physicsModel.cpp:16-20): NUC3D_RIEMANN_LF
     * (RiemannLF, :436-680), NUC3D_RIEMANN_AUSM (RiemannAUSM, :682-930) or
     * NUC3D_RIEMANN_AUSMP (RiemannAUSMp, :932-1179).  The quirk
     * NUC3D_QUIRK_ZETA_EIGEN belongs to RiemannLF only: the AUSM loops keep
     * each direction's own maximum eigenvalue. */
    int riemann;
    /* Method.in scheme_{x,y,z}_vis (fieldOperator.cpp:301-375): NUC3D_CD6
     * (centraldifference6th, the default), NUC3D_CD2 (centraldifference2nd)
     * or NUC3D_CD8 (centraldifference8th) per direction, for the velocity and
     * temperature gradients, the divergence of the viscous fluxes and the
     * statistics' gradients.  The halos are periodic whatever the inviscid
     * scheme (the reference hands these stencils the inviscid scheme's
     * bufferSize as their halo width, which cd8 outreaches with a 3-cell
     * scheme and cd6 with weno3js / upwind1st: there it reads outside its
     * data). */
    int vis_scheme[3];
} nuc3d_box_desc;
#define NUC3D_CD6 0
#define NUC3D_CD2 1
#define NUC3D_CD8 2
#define NUC3D_RIEMANN_LF 0
#define NUC3D_RIEMANN_AUSM 1
#define NUC3D_RIEMANN_AUSMP 2
#define NUC3D_FORCING_NONE 0
#define NUC3D_FORCING_CONST 1
#define NUC3D_FORCING_BAND 2

typedef struct nuc3d_ctx nuc3d_ctx;

/* Text of the last error on the calling thread ("" if none). */
NUC3D_API const char *nuc3d_last_error(void);
/* Version string of the library. */
NUC3D_API const char *nuc3d_version(void);

/* Fill *d with the reference decks' defaults (TGV-like: 64^3 2*pi box,
 * WENO5-JS, Navier-Stokes, Sutherland, Re 1000, M 0.5, Pr 0.72, gamma 1.4,
 * T_ref 110.4, T_inf 288, FP64, reference quirks) — physicsModel.cpp:23-64,
 * fieldOperator.cpp:22-32. */
NUC3D_API void nuc3d_box_desc_default(nuc3d_box_desc *d);

/* ---- whole-step solver (replaces block::solve's stage loop) --------------
 * One periodic box resident on the current device.  Replaces
 * NaiverStokesData3d::solve / EulerData3D::solve (NaiverStokes3d.cpp:37-73,
 * euler3d.cpp:260-277) + PDEData3d::solve (PDEData3d.cpp:155-176) +
 * tvdrk3rd (TVD-RK3.cpp:16-157) for the single-rank periodic case, with the
 * halo exchange (MPICommunicator.cpp:81-132) replaced by an in-kernel wrap. */
NUC3D_API int nuc3d_ctx_create(const nuc3d_box_desc *desc, void *stream, nuc3d_ctx **out);
NUC3D_API int nuc3d_ctx_destroy(nuc3d_ctx *ctx);
/* Bytes of device memory a context of this description holds. */
NUC3D_API long long nuc3d_ctx_bytes(const nuc3d_box_desc *desc);

/* State in/out (the 5 conserved fields rho, rho u, rho v, rho w, rho E).
 * Host variants copy through the context's stream and synchronise;
 * device variants are stream-ordered.  block.cpp:609-671 holds the same
 * five fields in its restart files. */
NUC3D_API int nuc3d_set_state_host(nuc3d_ctx *ctx, const double *const h_q[5]);
NUC3D_API int nuc3d_get_state_host(nuc3d_ctx *ctx, double *const h_q[5]);
/* The host copies enqueued on the context's stream without synchronising,
 * so that a caller advancing several contexts on their own streams overlaps
 * one context's copies with another's steps (the copy engines work in both
 * directions while the SMs compute).  The host arrays should be page-locked
 * (cudaHostAlloc / cudaHostRegister; pageable memory makes the copy
 * synchronous) and must stay valid and untouched until nuc3d_sync returns. */
NUC3D_API int nuc3d_set_state_host_async(nuc3d_ctx *ctx, const double *const h_q[5]);
NUC3D_API int nuc3d_get_state_host_async(nuc3d_ctx *ctx, double *const h_q[5]);
/* Copy lane (on != 0; off when a context is created): the context's host
 * transfers (the four host copies above) are issued one at a time per
 * direction together with those of every other context on the device whose
 * lane is on, in submission order.  Two large transfers in flight in the
 * same direction share the host link and both finish late; chained, each
 * one has the whole link, while uploads, downloads and the contexts' steps
 * still overlap.  A transfer waits for the previously submitted one and so
 * for whatever that one waits for on its own stream: turn the lane on for
 * contexts that take turns (a pipeline of steps through host memory), not
 * for independent ones.  No counterpart in the reference (one solver per
 * process, singleBlock.cpp:50-71). */
NUC3D_API int nuc3d_ctx_copy_lane(nuc3d_ctx *ctx, int on);
NUC3D_API int nuc3d_set_state_device(nuc3d_ctx *ctx, const double *const d_q[5]);
NUC3D_API int nuc3d_get_state_device(nuc3d_ctx *ctx, double *const d_q[5]);

/* Advance nsteps TVD-RK3 steps with dt = cfl * dt_local computed from the
 * state at each step's stage 0 (PDEData3d.cpp:161-165).  h_dt / h_res (host,
 * nsteps entries each, may be NULL) receive each step's dt and residual
 * (PDEData3d.cpp:178-213).  Synchronises only when h_dt or h_res is given. */
NUC3D_API int nuc3d_step(nuc3d_ctx *ctx, int nsteps, double cfl, double *h_dt, double *h_res);

/* Wait for the context's stream and report NUC3D_ERR_NONFINITE if any stage
 * produced a NaN/Inf state since the context was created (the reference has
 * no such check; physicsModel.cpp:340 masks negative pressure with fabs). */
NUC3D_API int nuc3d_sync(nuc3d_ctx *ctx);

/* One RHS evaluation of the current state (the NaiverStokesData3d::solve
 * part): d_rhs receives the 5 RHS fields (device), *h_dt_local the value the
 * reference passes to PDEData3d::setDt. */
NUC3D_API int nuc3d_rhs(nuc3d_ctx *ctx, double *const d_rhs[5], double *h_dt_local);

/* Kernel timing.  While enabled, every kernel nuc3d_step launches is
 * bracketed by CUDA events on the context's stream and the step waits for
 * them; nuc3d_profile_read adds up milliseconds and launch counts per kernel
 * class (NUC3D_PROF_* indices) since the last reset. */
#define NUC3D_PROF_PRIM 0      /* con2prim + max eigenvalue */
#define NUC3D_PROF_DT 1        /* dt from the eigenvalues */
#define NUC3D_PROF_VISC 2      /* CD6 gradients + viscous fluxes */
#define NUC3D_PROF_INV_X 3     /* inviscid sweep along x (WENO5 or CRWENO5) */
#define NUC3D_PROF_INV_Y 4
#define NUC3D_PROF_INV_Z 5
#define NUC3D_PROF_UPDATE 6    /* viscous divergence + RK stage */
#define NUC3D_PROF_RESIDUAL 7
#define NUC3D_PROF_CLASSES 8
NUC3D_API int nuc3d_profile_enable(nuc3d_ctx *ctx, int on);
NUC3D_API int nuc3d_profile_read(nuc3d_ctx *ctx, double *ms, long long *launches, int reset);
/* Kernels this context has launched since creation (all classes). */
NUC3D_API long long nuc3d_launch_count(const nuc3d_ctx *ctx);

/* ---- batches: many periodic boxes advanced together ----------------------
 * A batch holds boxes of any sizes, parameters and schemes (one precision
 * per batch) resident on the current device.  nuc3d_batch_step advances every
 * active box by nsteps TVD-RK3 steps, each box with its own dt (its own CFL
 * and eigenvalues), with one kernel launch per kernel class for all boxes; the
 * step is captured once as a CUDA graph and replayed.  Boxes may be added,
 * removed or (de)activated between steps (the next step rebuilds the work
 * lists and re-captures).  A box advanced in a batch gives the same result as
 * the same box advanced alone: no arithmetic crosses boxes.  This is the
 * batched form of the single-box solver; the reference runs one box per
 * process (singleBlock.cpp:50-71). */
typedef struct nuc3d_batch nuc3d_batch;
NUC3D_API int nuc3d_batch_create(int precision, void *stream, nuc3d_batch **out);
NUC3D_API int nuc3d_batch_destroy(nuc3d_batch *b);
/* Allocates the box's device memory (stream-ordered) and returns its id.
 * desc->precision must equal the batch's. */
NUC3D_API int nuc3d_batch_add(nuc3d_batch *b, const nuc3d_box_desc *desc, int *box_id);
NUC3D_API int nuc3d_batch_remove(nuc3d_batch *b, int box_id);
NUC3D_API int nuc3d_batch_set_active(nuc3d_batch *b, int box_id, int active);
NUC3D_API int nuc3d_batch_set_cfl(nuc3d_batch *b, int box_id, double cfl);
NUC3D_API int nuc3d_batch_set_state_host(nuc3d_batch *b, int box_id, const double *const h_q[5]);
NUC3D_API int nuc3d_batch_get_state_host(nuc3d_batch *b, int box_id, double *const h_q[5]);
NUC3D_API int nuc3d_batch_set_state_device(nuc3d_batch *b, int box_id,
                                           const double *const d_q[5]);
NUC3D_API int nuc3d_batch_get_state_device(nuc3d_batch *b, int box_id, double *const d_q[5]);
NUC3D_API int nuc3d_batch_step(nuc3d_batch *b, int nsteps);
/* dt and residual of the box's last n steps (n <= 1024; host arrays). */
NUC3D_API int nuc3d_batch_history(nuc3d_batch *b, int box_id, int n, double *h_dt,
                                  double *h_res);
NUC3D_API int nuc3d_batch_sync(nuc3d_batch *b);
NUC3D_API long long nuc3d_batch_box_steps(const nuc3d_batch *b, int box_id);
NUC3D_API double nuc3d_batch_time(nuc3d_batch *b, int box_id);
NUC3D_API int nuc3d_batch_profile_enable(nuc3d_batch *b, int on);
NUC3D_API int nuc3d_batch_profile_read(nuc3d_batch *b, double *ms, long long *launches,
                                       int reset);
NUC3D_API long long nuc3d_batch_launch_count(const nuc3d_batch *b);

/* Diagnostic, not part of the solver: the measured FMA-pipe throughput of
 * the current device in TFLOP/s (FP64 for NUC3D_FP64, FP32 for
 * NUC3D_MIXED), the roofline denominator of these stencil kernels (which run
 * on the FMA pipes, not on tensor cores, so neither a copy-bandwidth nor a
 * tensor-GEMM peak bounds them).  Runs a ~10 ms probe kernel on the
 * legacy stream; no solver entry point calls it. */
NUC3D_API int nuc3d_probe_peak(int precision, double *tflops);

/* Autotuner result.  The directional WENO sweep has variants in two tile
 * shapes: 32 cells along the sweep with runs of 1, 2 or 4 consecutive faces
 * per thread, and 64 cells with runs of 2 or 4 (fewer staged halo cells per
 * cell, twice the shared memory per block).  The first step after the set of
 * (scheme, direction) pairs changes times every variant on the live boxes and
 * keeps the fastest.  run_len[s*3+d] (s: the scheme id, NUC3D_WENO5JS ..
 * NUC3D_UPWIND1ST; d: x, y, z) receives the chosen run length (0 = not tuned;
 * always 0 for the line-solve schemes CRWENO5, hccs and hccs77, whose lines
 * have no run variants),
 * ms[(s*3+d)*3+v] the measured milliseconds per launch of the 32-cell
 * variants (run length 1, 2, 4).  run_len holds NUC3D_TUNING_SLOTS ints, ms
 * 3*NUC3D_TUNING_SLOTS doubles; either pointer may be NULL.
 * nuc3d_tuning_tiles: tile_cells[s*3+d] the chosen tile length (32 or 64; 0 =
 * not tuned), ms64[(s*3+d)*2+v] the milliseconds of the 64-cell variants
 * (run length 2, 4; 0 where not timed: mixed precision runs 32-cell tiles
 * only, because its FP32 staging is offset by each line's value at the
 * tile's first cell and another tile length would round differently);
 * NUC3D_TUNING_SLOTS ints and 2*NUC3D_TUNING_SLOTS doubles, either may be
 * NULL. */
#define NUC3D_TUNING_SLOTS 27
NUC3D_API int nuc3d_tuning(const nuc3d_ctx *ctx, int *run_len, double *ms);
NUC3D_API int nuc3d_batch_tuning(const nuc3d_batch *b, int *run_len, double *ms);
NUC3D_API int nuc3d_tuning_tiles(const nuc3d_ctx *ctx, int *tile_cells, double *ms64);
NUC3D_API int nuc3d_batch_tuning_tiles(const nuc3d_batch *b, int *tile_cells, double *ms64);
/* The other autotuned shape: the pencil depth of the 2.5-D stencil kernels
 * (viscous flux, update), i.e. how many z-planes one 32 x 8 column tile
 * marches (each tile re-reads a 6-plane halo, so deeper pencils read less but
 * make fewer, longer blocks).  The first step, and every step after the
 * batch's active cells have grown or shrunk past a factor 2 of those it was
 * tuned at, times one viscous-flux + update pass at each of
 * NUC3D_PENCIL_DEPTHS depths on the live boxes and keeps the fastest.
 * *depth receives the chosen depth (0 = not tuned), ms (3 doubles, may be
 * NULL) the measured milliseconds per pass for depths {32, 16, 64}. */
#define NUC3D_PENCIL_DEPTHS 3
NUC3D_API int nuc3d_tuning_pencil(const nuc3d_ctx *ctx, int *depth, double *ms);
NUC3D_API int nuc3d_batch_tuning_pencil(const nuc3d_batch *b, int *depth, double *ms);

/* ---- initial states generated on the device ------------------------------
 * NUC3D_INIT_TGV: block::initial_taylorgreen (block.cpp:359-395) on the cell
 *   centres with origin 0.
 * NUC3D_INIT_HIT: block::initial_hit (block.cpp:397-551): random-phase
 *   solenoidal velocity with E(k) ~ (k/k_peak)^4 exp(-2 (k/k_peak)^2), real
 *   part of the unnormalised backward transform, rescaled to
 *   u_rms = mach_t / (sqrt(3) M) (the reference writes mach_t / (sqrt(3) M^2);
 *   equal at M = 1); rho = 1, p = 1 / (gamma M^2).  The reference's phases
 *   come from an unseeded std::random_device; here phase c (0..2) of the mode
 *   at FFT index idx = i + nx (j + ny k) is output number 3 idx + c + 1 of the
 *   splitmix64 stream seeded with `seed`, times 2 pi, so a seed reproduces the
 *   field.  re_lambda > 0 sets the box's Reynolds number to
 *   re_lambda / (u_rms lambda), lambda the Taylor microscale of the generated
 *   field (postproc.cpp:871-872, spectral derivatives, rho = T = 1). */
#define NUC3D_INIT_TGV 1
#define NUC3D_INIT_HIT 2
typedef struct nuc3d_init_desc {
    int kind;                 /* NUC3D_INIT_TGV or NUC3D_INIT_HIT */
    unsigned long long seed;  /* HIT phase stream */
    double k_peak;            /* HIT spectrum peak wavenumber */
    double mach_t;            /* HIT turbulent Mach number */
    double re_lambda;         /* HIT: > 0 sets the Reynolds number from it */
} nuc3d_init_desc;
/* h_info (3 doubles, may be NULL): u_rms, Taylor microscale, the box's
 * Reynolds number after the call (NaN for the first two with TGV). */
NUC3D_API int nuc3d_init_state(nuc3d_ctx *ctx, const nuc3d_init_desc *init, double *h_info);
NUC3D_API int nuc3d_batch_init_state(nuc3d_batch *b, int box_id, const nuc3d_init_desc *init,
                                     double *h_info);

/* ---- serving: a request loop over a batch ---------------------------------
 * No counterpart in the reference, which runs one solve per process
 * (NUC3d.cpp main -> singleBlock::solve).  A server owns one batch (one
 * precision) on the device current at creation and one worker thread.
 * nuc3d_serve_submit queues a solve from any thread.  The worker admits
 * queued solves in submission order while the sum of the resident solves'
 * device bytes (nuc3d_ctx_bytes of each) fits the budget and fewer than
 * max_resident are resident; it allocates the box, uploads h_q0 or generates
 * the initial state, and advances all resident solves together in chunks of
 * steps (the batch's CUDA graph replayed; a chunk is no longer than the
 * shortest remaining solve and about chunk_ms long, its step time predicted
 * from the last chunk's device time per resident cell), so solves join and leave
 * the running batch between chunks (continuous batching).  A finished solve's
 * state is copied to h_q_out, its memory released and its result posted.
 * A solve gives the same final state alone and in any mix: no arithmetic
 * crosses boxes and every kernel variant rounds identically. */
typedef struct nuc3d_server nuc3d_server;

typedef struct nuc3d_serve_config {
    int precision;            /* NUC3D_FP64 or NUC3D_MIXED */
    long long budget_bytes;   /* device bytes for resident solves; <= 0: 90 % of free */
    int max_resident;         /* <= 0: 256 */
    int max_chunk_steps;      /* <= 0: 64 */
    double chunk_ms;          /* target device time of one chunk; <= 0: 20 ms */
} nuc3d_serve_config;

typedef struct nuc3d_solve_request {
    nuc3d_box_desc desc;      /* precision is replaced by the server's */
    int nsteps;               /* TVD-RK3 steps */
    double cfl;
    nuc3d_init_desc init;     /* init.kind 0: the state comes from h_q0 */
    const double *h_q0[5];    /* host; must stay valid until the result is collected */
    double *h_q_out[5];       /* host, written at completion (all NULL: not copied) */
    long long tag;            /* returned in the result */
} nuc3d_solve_request;

typedef struct nuc3d_solve_result {
    long long ticket, tag;
    int status;               /* NUC3D_OK or the solve's error code */
    int pad;
    long long steps, cells;
    double sim_time, dt_last, res_last;
    double reynolds;          /* Reynolds number the solve ran with */
    double t_submit, t_admit, t_done;  /* seconds on the server's clock */
    char error[160];
} nuc3d_solve_result;

typedef struct nuc3d_serve_stats {
    long long submitted, completed, failed;
    int queued, resident, peak_resident, pad;
    long long resident_bytes, peak_resident_bytes, budget_bytes;
    long long batch_steps, chunks, cell_updates, launches;
    long long graph_captures; /* CUDA-graph captures of the batch step (one per
                                 change of the resident set that is stepped) */
    double busy_s;            /* wall time spent advancing resident solves */
    double now_s;             /* the server's clock */
} nuc3d_serve_stats;

NUC3D_API void nuc3d_serve_config_default(nuc3d_serve_config *cfg);
NUC3D_API int nuc3d_serve_create(const nuc3d_serve_config *cfg, nuc3d_server **out);
/* Cancels queued and resident solves (status NUC3D_ERR_CANCELLED) and joins
 * the worker. */
NUC3D_API int nuc3d_serve_destroy(nuc3d_server *s);
NUC3D_API int nuc3d_serve_submit(nuc3d_server *s, const nuc3d_solve_request *req,
                                 long long *ticket);
/* Waits for solve `ticket` (ticket < 0: the next solve to finish) and
 * collects its result; timeout_s < 0 waits without limit. */
NUC3D_API int nuc3d_serve_wait(nuc3d_server *s, long long ticket, double timeout_s,
                               nuc3d_solve_result *out);
NUC3D_API int nuc3d_serve_info(nuc3d_server *s, nuc3d_serve_stats *out);

/* ---- turbulence statistics on the device (FP64) ---------------------------
 * postproc::solveQ (postproc.cpp:736-930) of the box's current state, single
 * rank: CD6 velocity gradients of the primitives, then the 16 averages of
 * enstrophy.dat (indices 0..15: du/dx, du/dy, du/dz, dv/dx, dv/dy, dv/dz,
 * dw/dx, dw/dy, dw/dz, omega_x, omega_y, omega_z, enstrophy |omega|^2/2,
 * Q, helicity, kinetic energy rho|u|^2/2) and the 9 values of turb_para.dat
 * (16..24: u_rms, turbulent Mach, sqrt(<(du_i/dx_i)^2>/3), mean Sutherland
 * viscosity, Re_lambda, Taylor microscale, mean density, eddy turnover time,
 * velocity-derivative skewness).  Index 25, not in the reference: the viscous
 * dissipation <mu (|omega|^2 + 4/3 (div u)^2)> with the box's viscosity model.
 * Synchronises; h_out receives NUC3D_STATS doubles. */
#define NUC3D_STATS 26
#define NUC3D_STAT_ENSTROPHY 12
#define NUC3D_STAT_KINETIC 15
#define NUC3D_STAT_U_RMS 16
#define NUC3D_STAT_MACH_T 17
#define NUC3D_STAT_RE_LAMBDA 20
#define NUC3D_STAT_LAMBDA 21
#define NUC3D_STAT_SKEWNESS 24
#define NUC3D_STAT_DISSIPATION 25
NUC3D_API int nuc3d_stats(nuc3d_ctx *ctx, double *h_out);
NUC3D_API int nuc3d_batch_stats(nuc3d_batch *b, int box_id, double *h_out);

/* Shell-binned spectra of the current state: postproc::solveFFT
 * (postproc.cpp:931-1184) with fft.cpp:182-572, FP64, FFTs by cuFFT.
 * h_out receives NUC3D_SPECTRA rows of kmax shells (row-major), kmax =
 * min(nx, ny, nz)/2 written to *kmax; h_out may be NULL to query kmax.
 * Rows, as the reference's power_shell_<step>_<name>.dat files:
 *   kin, kinc, kins, kinl, kinr: 0.5 |u^|^2 of the velocity transform (normalised
 *     by 1/N) and of its compressive, solenoidal and left/right helical parts,
 *     binned over the folded |k| with |k| = 1 at k = 0 (the mean flow falls in
 *     shell 1, shell 0 stays empty);
 *   hel, ens, den, pre: |f^|^2 of the helicity field w.u, the enstrophy field
 *     |w|^2/2, density and pressure, binned as fft.cpp:517-531 does: over the
 *     unfolded i^2 + j^2 + k^2 (only the non-negative octant of wavenumbers).
 * Shell i holds |k| in (i - 1/2, i + 1/2].  Allocates 112 bytes per cell of
 * scratch for the call and synchronises the context's stream. */
#define NUC3D_SPECTRA 9
#define NUC3D_SPEC_KIN 0
#define NUC3D_SPEC_KINC 1
#define NUC3D_SPEC_KINS 2
#define NUC3D_SPEC_KINL 3
#define NUC3D_SPEC_KINR 4
#define NUC3D_SPEC_HEL 5
#define NUC3D_SPEC_ENS 6
#define NUC3D_SPEC_DEN 7
#define NUC3D_SPEC_PRE 8
NUC3D_API int nuc3d_spectra(nuc3d_ctx *ctx, double *h_out, int *kmax);
NUC3D_API int nuc3d_batch_spectra(nuc3d_batch *b, int box_id, double *h_out, int *kmax);

/* Simulated time advanced by this context so far (block.cpp:208-209). */
NUC3D_API double nuc3d_ctx_time(const nuc3d_ctx *ctx);

/* ---- per-operator entry points (the reference's scheme plug-in API) -------
 * These mirror the `interoplation`, `differential` and `integration`
 * interfaces (fieldOperator.h:13-81) on device buffers, so a reference-side
 * subclass can forward to them; halos are explicit, as in the reference.
 *
 * nuc3d_reconstruct = interpolationInner + interpolationBoundaryL +
 *   interpolationBoundaryR of weno5js (weno5js.cpp:19-628), weno5z
 *   (weno5z.cpp:18-637), crweno5 (crweno5.cpp:25-837) with tilesize 3, or
 *   weno7js (weno7js.cpp:17-824) or hccs (hccs.cpp) with tilesize 4.
 *   Along the fastest axis of an (nx,ny,nz) field; halo_l/halo_r are (h,ny,nz)
 *   with h = 4 for weno7js and hccs and 3 otherwise (the received MPI buffers,
 *   bufferData.cpp:16-47); out is (nx+1,ny,nz),
 *   face m between cells m-1 and m.  upwind = +1 or -1.  crweno5 needs
 *   nx <= 4096.  quirks: NUC3D_QUIRK_WENOZ_BETA2 is honoured. */
NUC3D_API int nuc3d_reconstruct(int scheme, int upwind, unsigned quirks, int nx, int ny, int nz,
                      const double *d_in, const double *d_halo_l, const double *d_halo_r,
                      double *d_out, void *stream);

/* CRWENO5 reconstruction that allocates nothing.  No counterpart in the
 * reference: it exists for callers that cannot let a library allocate device
 * memory (a host code that owns all device memory through its own pool, or
 * a plug-in called where allocation is forbidden).  Same arguments and
 * results as nuc3d_reconstruct(NUC3D_CRWENO5, ...), but the Thomas-sweep
 * scratch is a fixed 4 MiB array in the library's device image (held by
 * every GPU that loads the library until exit), so 2*nx*ny*nz must not
 * exceed 524288 (and nx must not exceed 4096, as for nuc3d_reconstruct);
 * larger calls return NUC3D_ERR_INVALID.  Every call looks up the array's
 * address on the current device (cudaGetSymbolAddress, which allocates
 * nothing), so a device reset in the same process is harmless; the first
 * call on each device also loads the library's device code there and should
 * come before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race and must be serialised. */
NUC3D_API int nuc3d_reconstruct_crweno5_noalloc(int upwind, int nx, int ny, int nz,
                                                const double *d_in, const double *d_halo_l,
                                                const double *d_halo_r, double *d_out,
                                                void *stream);

/* centraldifference6th::differentialInner + BoundaryL + BoundaryR
 * (centraldifference6th.cpp:16-186); out is (nx,ny,nz). */
NUC3D_API int nuc3d_cd6(int nx, int ny, int nz, double dx, const double *d_in, const double *d_halo_l,
              const double *d_halo_r, double *d_out, void *stream);

/* The `differential` plug-in of any registered scheme (fieldOperator.h:58-81):
 * scheme NUC3D_CD6, NUC3D_CD2 or NUC3D_CD8 (centraldifference6th.cpp:16-186,
 * centraldifference2nd.cpp:16-146, centraldifference8th.cpp:22-205) with the
 * reference's tilesize `tile` (the inviscid scheme's bufferSize, 1..4): the
 * halos are (tile,ny,nz) and cd8's cells within `tile` of a line end take its
 * boundary form.  NUC3D_ERR_INVALID where the stencil would reach past the
 * halo (cd6 with tile < 3, cd8 with tile < 4), nx < 2 tile or nx > 4096. */
NUC3D_API int nuc3d_differential(int scheme, int tile, int nx, int ny, int nz, double dx,
                                 const double *d_in, const double *d_halo_l,
                                 const double *d_halo_r, double *d_out, void *stream);

/* tvdrk3rd::integrationAll (TVD-RK3.cpp:16-157): d_ui updated in place from
 * d_rhs (the RHS R, dQ/dt = -R), d_un (u_n), stage 0..2. */
NUC3D_API int nuc3d_tvdrk3_stage(int stage, long long n, double dt, const double *const d_rhs[5],
                       const double *const d_un[5], double *const d_ui[5], void *stream);

#ifdef __cplusplus
}
#endif
#endif /* NUC3D_B200_H */
