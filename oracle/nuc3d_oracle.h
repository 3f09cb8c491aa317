/*
 * CPU restatement of NUC3d's RHS evaluation and TVD-RK3 step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle that the CUDA path is checked
 * against; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it.  The product never links or calls it.
 *
 * Pinned against the reference's own translation units (oracle/_ref, built by
 * `make -C oracle ref` from the reference sources) through the golden fixtures
 * in tests/golden/ (bitwise equality expected: both sides are strict-IEEE
 * FP64 on the host, with the reference's operation order restated here).
 *
 * All fields are FP64, x-fastest: idx = i + nx*(j + ny*k), the layout of the
 * reference's Field (field.h, block.cpp:119).  The reference's rotated
 * per-direction copies (euler3d.cpp:71-76) are pure data movement and are not
 * reproduced: lines are walked with strides instead.
 */
#ifndef NUC3D_ORACLE_H
#define NUC3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* scheme ids (fieldOperator.cpp:152-166 strings weno5js / weno5z / crweno5) */
enum { OR_WENO5JS = 0, OR_WENO5Z = 1, OR_CRWENO5 = 2, OR_WENO7 = 3, OR_HCCS = 4, OR_HCCS77 = 5,
       OR_HCCS78 = 6, OR_WENO3JS = 7, OR_UPWIND1 = 8 };
/* viscosity models (physicsModel.cpp:44-49; power law is an extra model) */
enum { OR_SUTHERLAND = 0, OR_CONSTANT = 1, OR_POWERLAW = 2 };
/* differential schemes: Method.in scheme_*_vis "cd6", "cd2", "cd8"
 * (fieldOperator.cpp:301-375; any other string is cd6) */
enum { OR_CD6 = 0, OR_CD2 = 1, OR_CD8 = 2 };

/* Reference behaviours that look like defects; each is reproduced when its
 * bit is set (the default, OR_QUIRKS_REFERENCE) and replaced by the textbook
 * form when cleared. */
enum {
    OR_Q_ZETA_EIGEN = 1u << 0,   /* physicsModel.cpp:653-654: z eigen folded into eta, z = 0 */
    OR_Q_WENOZ_BETA2 = 1u << 1,  /* weno5z.cpp:80: inner '+' beta2 uses f[i+1] twice */
    OR_Q_OFFDIAG_DIV = 1u << 2,  /* NaiverStokes3d.cpp:267-270: -2/3 div(u) on off-diagonals */
    OR_Q_FABS_PRESSURE = 1u << 3,/* physicsModel.cpp:340: p = |(E - rho|u|^2/2)(gamma-1)| */
    OR_Q_CRWENO_BOUNDED = 1u << 4,/* crweno5.cpp:45-402: bounded line system, explicit ends */
};
#define OR_QUIRKS_REFERENCE 0x1fu

typedef struct {
    int nx, ny, nz;
    double dx, dy, dz;
    int scheme[3];      /* per direction */
    int navier_stokes;  /* 1: NavierStokes3d, 0: Euler3d (block.cpp:146-157) */
    int visc_model;
    double gamma, mach, reynolds, prandtl, t_ref, t_inf, powerlaw_exp;
    unsigned quirks;
    int riemann;        /* OR_LF, OR_AUSM, OR_AUSMP: PhysModel.in RiemannSolver */
    int vis[3];         /* OR_CD6, OR_CD2, OR_CD8 per direction: scheme_*_vis */
} or_box;

/* flux splittings (physicsModel.cpp:16-20 map "LF", "AUSM", "AUSMp") */
enum { OR_LF = 0, OR_AUSM = 1, OR_AUSMP = 2 };

/* physicsModel::con2prim.  prim: rho,u,v,w,p,T,e,c (8 fields). */
void or_con2prim(const or_box *b, const double *const q[5], double *const prim[8]);

/* physicsModel::RiemannLF for one direction d (0,1,2).  fl/fr: F+ / F- per
 * equation, x-fastest.  *eig receives the running maxEigen this direction's
 * loop produces; with OR_Q_ZETA_EIGEN the z loop updates eig_eta instead. */
void or_lf_split(const or_box *b, const double *const q[5], const double *const prim[8],
                 double *const fl[3][5], double *const fr[3][5], double eig[3]);

/* physicsModel::RiemannAUSM / RiemannAUSMp (physicsModel.cpp:682-1278), the
 * point-wise Mach-number splittings, same layout as or_lf_split.  No
 * eigenvalue quirk: each direction's loop updates its own maxEigen. */
void or_ausm_split(const or_box *b, const double *const q[5], const double *const prim[8],
                   double *const fl[3][5], double *const fr[3][5], double eig[3]);

/* The reference's per-field reconstruction interface
 * (interpolationInner + BoundaryL + BoundaryR): along the fastest axis of an
 * (nx,ny,nz) field with explicit halos of the scheme's buffer width (3 for
 * the 5-point schemes, 4 for OR_WENO7; fieldOperator.cpp:128-175), shaped
 * (width,ny,nz); out is (nx+1,ny,nz).  Widths: 3 for the 5-point schemes, 4
 * for OR_WENO7 and OR_HCCS. */
int or_reconstruct_field(int scheme, int upwind, unsigned quirks, int nx, int ny, int nz,
                         const double *in, const double *halo_l, const double *halo_r,
                         double *out);

/* centraldifference6th, same field/halo convention; out is (nx,ny,nz). */
int or_cd6_field(int nx, int ny, int nz, double dx, const double *in, const double *halo_l,
                 const double *halo_r, double *out);

/* differentialInner + differentialBoundaryL/R of the scheme (OR_CD6, OR_CD2,
 * OR_CD8) with the reference's tilesize `tile` (1..4): halos are (tile,ny,nz)
 * and cells within `tile` of a line end take the boundary form.  -1 for cd8
 * with tile < 4 (the reference's stencil reads outside its data there). */
int or_cd_field(int scheme, int tile, int nx, int ny, int nz, double dx, const double *in,
                const double *halo_l, const double *halo_r, double *out);

/* tvdrk3rd::integrationAll on n cells, ui updated in place. */
void or_rk3_stage(int stage, long n, double dt, const double *const rhs[5],
                  const double *const un[5], double *const ui[5]);

/* One RHS evaluation (NaiverStokesData3d::solve or EulerData3D::solve) of a
 * fully periodic box.  Returns dt_local (euler3d.cpp:459-466). */
double or_rhs(const or_box *b, const double *const q[5], double *const rhs[5]);

/* nsteps TVD-RK3 steps in place; dt[s], res[s] per step (block.cpp:191-215,
 * PDEData3d.cpp:155-213). */
void or_run_steps(const or_box *b, double cfl, int nsteps, double *const q[5], double *dt,
                  double *res);

/* postproc::solveQ (postproc.cpp:736-930) of a periodic box, single rank:
 *   out[0..15]  the averages written to enstrophy.dat: du/dx, du/dy, du/dz,
 *               dv/dx .. dw/dz, omega0..2, enstrophy, Q, helicity, kinetic
 *   out[16..24] turb_para.dat: u_rms, Mt, sqrt(div_aver), mu_aver,
 *               Re_lambda, lambda, rho_bar, tau_t, skewness
 *   out[25]     viscous dissipation <mu (|omega|^2 + 4/3 (div u)^2)>, mu of
 *               the box's viscosity model (not in the reference) */
#define OR_NSTATS 26
void or_stats(const or_box *b, const double *const q[5], double out[OR_NSTATS]);

/* Taylor-Green initial state (block.cpp:103-140, 359-395); x0,y0,z0 origin. */
void or_init_tgv(const or_box *b, double x0, double y0, double z0, double *const q[5]);

#ifdef __cplusplus
}
#endif
#endif
