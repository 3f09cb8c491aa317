/*
 * CPU restatement of NUC3d's RHS evaluation and TVD-RK3 step.
 *
 * TEST INFRASTRUCTURE ONLY (see nuc3d_oracle.h).  Every function cites the
 * reference file:line whose arithmetic it restates.  Operation order follows
 * the reference expression by expression so that, compiled with strict IEEE
 * FP64 (no -ffast-math, no FMA contraction on x86-64), the results are
 * bitwise identical to the reference's own code.  Two details matter for
 * that:
 *   - the reference writes squares two ways.  std::pow(x, 2) with a literal
 *     exponent is folded to x*x by the compiler; std::pow(x, p) with the
 *     scheme's int member p is a libm pow() call, which differs from x*x by
 *     one ulp for about 0.1% of inputs.  SQ() and PW() below keep them apart.
 *   - Sutherland's T^1.5 is libm pow(T, 1.5) (physicsModel.cpp:220).
 *
 * The RHS and the RK stage run their independent lines and cells on POSIX
 * threads (NUC3D_ORACLE_THREADS, default: the online cores).  Every line and
 * cell is computed exactly as in a serial run, the running maxima are
 * combined with fmax (associative; it ignores a NaN operand in any order)
 * and the residual sum stays serial, so the results are bitwise the same for
 * any thread count.
 */
#define _POSIX_C_SOURCE 200809L
#include "nuc3d_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* The reference's schemes hold p = 2 as a runtime member (weno5js.cpp:9,
 * weno5z.cpp:8, crweno5.cpp:15).  Keeping it in a global stops the compiler
 * from folding pow(x, p) into x*x, as it cannot in the reference. */
int or_weno_p = 2;

#define SQ(x) ((x) * (x))
#define PW(x) pow((x), (double)or_weno_p)

/* ------------------------------------------------------------ threads ---- */

#define OR_MAX_THREADS 64

typedef void (*or_range_fn)(void *ctx, int part, long lo, long hi);

typedef struct {
    or_range_fn fn;
    void *ctx;
    int part;
    long lo, hi;
} or_task;

static int or_thread_count(void) {
    const char *e = getenv("NUC3D_ORACLE_THREADS");
    long t = e ? atol(e) : sysconf(_SC_NPROCESSORS_ONLN);
    if (t < 1) t = 1;
    if (t > OR_MAX_THREADS) t = OR_MAX_THREADS;
    return (int)t;
}

static void *or_task_main(void *arg) {
    or_task *t = (or_task *)arg;
    t->fn(t->ctx, t->part, t->lo, t->hi);
    return NULL;
}

/* Runs fn over [0, n) in contiguous parts, one per thread (part 0 on the
 * calling thread; a part whose thread cannot be started runs on the calling
 * thread too).  Returns the number of parts. */
static int or_parallel(long n, or_range_fn fn, void *ctx) {
    int T = or_thread_count();
    if (n < T) T = n > 0 ? (int)n : 1;
    or_task task[OR_MAX_THREADS];
    pthread_t th[OR_MAX_THREADS];
    int started[OR_MAX_THREADS] = {0};
    for (int i = 0; i < T; ++i) {
        task[i].fn = fn;
        task[i].ctx = ctx;
        task[i].part = i;
        task[i].lo = n * i / T;
        task[i].hi = n * (i + 1) / T;
    }
    for (int i = 1; i < T; ++i) started[i] = pthread_create(&th[i], NULL, or_task_main, &task[i]) == 0;
    or_task_main(&task[0]);
    for (int i = 1; i < T; ++i) {
        if (started[i])
            pthread_join(th[i], NULL);
        else
            or_task_main(&task[i]);
    }
    return T;
}

/* schemes.hpp:14-36 */
static const double A[3][3] = {{1.0 / 3.0, -7.0 / 6.0, 11.0 / 6.0},
                               {-1.0 / 6.0, 5.0 / 6.0, 1.0 / 3.0},
                               {1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0}};
static const double C_W5[3] = {0.1, 0.6, 0.3};
static const double C_CR5[3] = {0.2, 0.5, 0.3};
static const double G0 = 13.0 / 12.0;
static const double G1 = 1.0 / 4.0;
static const double CD6[3] = {3.0 / 4.0, -3.0 / 20.0, 1.0 / 60.0};
static const double CD8[4] = {4.0 / 5.0, -1.0 / 5.0, 4.0 / 105.0, -1.0 / 280.0}; /* schemes.hpp:36 */

/* ---------------------------------------------------------------- WENO5 --- */

/* WENO3-JS on an upwind-oriented stencil g[0..2] (weno3js.cpp:79-93 for '+',
 * :134-148 for '-', and the halo forms): eps = 1e-6, linear weights 1/3,
 * 2/3; the indicators square with a literal std::pow(x, 2) (x*x), the
 * weights raise to the member p = 2 through libm's pow. */
static double weno3js_face(const double g[3]) {
    const double ss = 1.0e-6;
    double is0 = SQ(g[0] - g[1]);
    double is1 = SQ(g[1] - g[2]);
    double q20 = -0.5 * g[0] + 1.5 * g[1];
    double q21 = 0.5 * g[1] + 0.5 * g[2];
    double aa0 = 1.0 / 3.0 / PW(ss + is0);
    double aa1 = 2.0 / 3.0 / PW(ss + is1);
    double w0 = aa0 / (aa0 + aa1);
    double w1 = aa1 / (aa0 + aa1);
    return w0 * q20 + w1 * q21;
}

/* WENO5-JS on an upwind-oriented stencil f[0..4] (f[0] farthest upwind).
 * weno5js.cpp:75-108 (inner +), :156-189 (inner -), :275-308 (halo forms);
 * all four are this expression on differently gathered stencils.  eps=1e-6. */
static double weno5js_face(const double f[5]) {
    const double ss = 1.0e-6;
    double is0 = G0 * SQ(f[0] - 2.0 * f[1] + f[2]) + G1 * SQ(f[0] - 4.0 * f[1] + 3.0 * f[2]);
    double is1 = G0 * SQ(f[1] - 2.0 * f[2] + f[3]) + G1 * SQ(f[1] - f[3]);
    double is2 = G0 * SQ(f[2] - 2.0 * f[3] + f[4]) + G1 * SQ(3.0 * f[2] - 4.0 * f[3] + f[4]);
    double q30 = A[0][0] * f[0] + A[0][1] * f[1] + A[0][2] * f[2];
    double q31 = A[1][0] * f[1] + A[1][1] * f[2] + A[1][2] * f[3];
    double q32 = A[2][0] * f[2] + A[2][1] * f[3] + A[2][2] * f[4];
    double alpha0 = C_W5[0] / PW(ss + is0);
    double alpha1 = C_W5[1] / PW(ss + is1);
    double alpha2 = C_W5[2] / PW(ss + is2);
    double alphaSum = alpha0 + alpha1 + alpha2;
    double omega0 = alpha0 / alphaSum;
    double omega1 = alpha1 / alphaSum;
    double omega2 = alpha2 / alphaSum;
    return omega0 * q30 + omega1 * q31 + omega2 * q32;
}

/* WENO5-Z, weno5z.cpp:74-109 and the halo forms :275-310.  eps=1e-40.
 * beta2_quirk reproduces weno5z.cpp:80 (inner '+' only): the first term of
 * beta2 reads f[i]-2f[i+1]+f[i+1] instead of f[i]-2f[i+1]+f[i+2]. */
static double weno5z_face(const double f[5], int beta2_quirk) {
    const double ss = 1.0e-40;
    double is0 = G0 * PW(f[0] - 2.0 * f[1] + f[2]) + G1 * PW(f[0] - 4.0 * f[1] + 3.0 * f[2]);
    double is1 = G0 * PW(f[1] - 2.0 * f[2] + f[3]) + G1 * PW(f[1] - f[3]);
    double is2 = beta2_quirk
                     ? G0 * PW(f[2] - 2.0 * f[3] + f[3]) + G1 * PW(3.0 * f[2] - 4.0 * f[3] + f[4])
                     : G0 * PW(f[2] - 2.0 * f[3] + f[4]) + G1 * PW(3.0 * f[2] - 4.0 * f[3] + f[4]);
    double q30 = A[0][0] * f[0] + A[0][1] * f[1] + A[0][2] * f[2];
    double q31 = A[1][0] * f[1] + A[1][1] * f[2] + A[1][2] * f[3];
    double q32 = A[2][0] * f[2] + A[2][1] * f[3] + A[2][2] * f[4];
    double tau = fabs(is2 - is0);
    double alpha0 = C_W5[0] * (1.0 + PW(tau / (is0 + ss)));
    double alpha1 = C_W5[1] * (1.0 + PW(tau / (is1 + ss)));
    double alpha2 = C_W5[2] * (1.0 + PW(tau / (is2 + ss)));
    double alphaSum = alpha0 + alpha1 + alpha2;
    double omega0 = alpha0 / alphaSum;
    double omega1 = alpha1 / alphaSum;
    double omega2 = alpha2 / alphaSum;
    return omega0 * q30 + omega1 * q31 + omega2 * q32;
}

/* schemes.hpp:21-31 */
static const double A7[4][4] = {{-3.0 / 12.0, 13.0 / 12.0, -23.0 / 12.0, 25.0 / 12.0},
                                {1.0 / 12.0, -5.0 / 12.0, 13.0 / 12.0, 3.0 / 12.0},
                                {-1.0 / 12.0, 7.0 / 12.0, 7.0 / 12.0, -1.0 / 12.0},
                                {3.0 / 12.0, 13.0 / 12.0, -5.0 / 12.0, 1.0 / 12.0}};
static const double C_W7[4] = {1.0 / 35.0, 12.0 / 35.0, 18.0 / 35.0, 4.0 / 35.0};

/* The reference's weno7js: weno7js.cpp:79-126 (inner +), :179-226 (inner -),
 * :316-371 and the other halo forms, all this expression on an
 * upwind-oriented 7-cell stencil f[0..6].  Its weights are the Z form
 * alpha_k = c_k (1 + (tau7/(eps+beta_k))^p), tau7 = |beta0 - beta3|,
 * eps = 1e-20 (weno7js.cpp:14, :111-114; the JS form is commented out). */
static double weno7_face_eps(const double f[7], double ss, int literal_square);
static double weno7_face(const double f[7]) { return weno7_face_eps(f, 1.0e-20, 0); }

/* The same face with the caller's eps and squaring: hccs evaluates its WENO7
 * faces with its own member ss = 1e-40 (hccs.cpp:13-17) and squares with
 * std::pow(x, 2), a literal exponent the compiler turns into x*x, where
 * weno7js raises to its runtime member p through libm's pow. */
static double weno7_face_eps(const double f[7], double ss, int literal_square) {
    double is0 = f[0] * (547.0 * f[0] - 3882.0 * f[1] + 4642.0 * f[2] - 1854.0 * f[3]) +
                 f[1] * (7043.0 * f[1] - 17246.0 * f[2] + 7042.0 * f[3]) +
                 f[2] * (11003.0 * f[2] - 9402.0 * f[3]) + 2107.0 * f[3] * f[3];
    double is1 = f[1] * (267.0 * f[1] - 1642.0 * f[2] + 1602.0 * f[3] - 494.0 * f[4]) +
                 f[2] * (2843.0 * f[2] - 5966.0 * f[3] + 1922.0 * f[4]) +
                 f[3] * (3443.0 * f[3] - 2522.0 * f[4]) + 547.0 * f[4] * f[4];
    double is2 = f[2] * (547.0 * f[2] - 2522.0 * f[3] + 1922.0 * f[4] - 494.0 * f[5]) +
                 f[3] * (3443.0 * f[3] - 5966.0 * f[4] + 1602.0 * f[5]) +
                 f[4] * (2843.0 * f[4] - 1642.0 * f[5]) + 267.0 * f[5] * f[5];
    double is3 = f[3] * (2107.0 * f[3] - 9402.0 * f[4] + 7042.0 * f[5] - 1854.0 * f[6]) +
                 f[4] * (11003.0 * f[4] - 17246.0 * f[5] + 4642.0 * f[6]) +
                 f[5] * (7043.0 * f[5] - 3882.0 * f[6]) + 547.0 * f[6] * f[6];
    double q40 = A7[0][0] * f[0] + A7[0][1] * f[1] + A7[0][2] * f[2] + A7[0][3] * f[3];
    double q41 = A7[1][0] * f[1] + A7[1][1] * f[2] + A7[1][2] * f[3] + A7[1][3] * f[4];
    double q42 = A7[2][0] * f[2] + A7[2][1] * f[3] + A7[2][2] * f[4] + A7[2][3] * f[5];
    double q43 = A7[3][0] * f[3] + A7[3][1] * f[4] + A7[3][2] * f[5] + A7[3][3] * f[6];
    double tau7 = fabs(is0 - is3);
    double r0 = tau7 / (ss + is0), r1 = tau7 / (ss + is1), r2 = tau7 / (ss + is2),
           r3 = tau7 / (ss + is3);
    double alpha0 = C_W7[0] * (1.0 + (literal_square ? SQ(r0) : PW(r0)));
    double alpha1 = C_W7[1] * (1.0 + (literal_square ? SQ(r1) : PW(r1)));
    double alpha2 = C_W7[2] * (1.0 + (literal_square ? SQ(r2) : PW(r2)));
    double alpha3 = C_W7[3] * (1.0 + (literal_square ? SQ(r3) : PW(r3)));
    double alphaSum = alpha0 + alpha1 + alpha2 + alpha3;
    double omega0 = alpha0 / alphaSum;
    double omega1 = alpha1 / alphaSum;
    double omega2 = alpha2 / alphaSum;
    double omega3 = alpha3 / alphaSum;
    return omega0 * q40 + omega1 * q41 + omega2 * q42 + omega3 * q43;
}

/* schemes.hpp:30 coeff_upwindcompact_c */
static const double C_UPC[3] = {2.0 / 7.0, 4.0 / 7.0, 1.0 / 7.0};

/* The WENO7-Z face of hccs77 and hccs78 (hccs77.cpp:79-135, hccs78.cpp:81-139
 * and their halo forms): eps = 1e-20 (their member ss, :14), squares through
 * libm's pow with their runtime member p = 2, as weno7js.  Also returns the
 * unnormalised weights' sum, from which both form their blend
 * theta = 1/(1 + (sum alpha - 1)^p). */
static double weno7z_face_sum(const double f[7], double *alpha_sum) {
    const double ss = 1.0e-20;
    double is0 = f[0] * (547.0 * f[0] - 3882.0 * f[1] + 4642.0 * f[2] - 1854.0 * f[3]) +
                 f[1] * (7043.0 * f[1] - 17246.0 * f[2] + 7042.0 * f[3]) +
                 f[2] * (11003.0 * f[2] - 9402.0 * f[3]) + 2107.0 * f[3] * f[3];
    double is1 = f[1] * (267.0 * f[1] - 1642.0 * f[2] + 1602.0 * f[3] - 494.0 * f[4]) +
                 f[2] * (2843.0 * f[2] - 5966.0 * f[3] + 1922.0 * f[4]) +
                 f[3] * (3443.0 * f[3] - 2522.0 * f[4]) + 547.0 * f[4] * f[4];
    double is2 = f[2] * (547.0 * f[2] - 2522.0 * f[3] + 1922.0 * f[4] - 494.0 * f[5]) +
                 f[3] * (3443.0 * f[3] - 5966.0 * f[4] + 1602.0 * f[5]) +
                 f[4] * (2843.0 * f[4] - 1642.0 * f[5]) + 267.0 * f[5] * f[5];
    double is3 = f[3] * (2107.0 * f[3] - 9402.0 * f[4] + 7042.0 * f[5] - 1854.0 * f[6]) +
                 f[4] * (11003.0 * f[4] - 17246.0 * f[5] + 4642.0 * f[6]) +
                 f[5] * (7043.0 * f[5] - 3882.0 * f[6]) + 547.0 * f[6] * f[6];
    double q40 = A7[0][0] * f[0] + A7[0][1] * f[1] + A7[0][2] * f[2] + A7[0][3] * f[3];
    double q41 = A7[1][0] * f[1] + A7[1][1] * f[2] + A7[1][2] * f[3] + A7[1][3] * f[4];
    double q42 = A7[2][0] * f[2] + A7[2][1] * f[3] + A7[2][2] * f[4] + A7[2][3] * f[5];
    double q43 = A7[3][0] * f[3] + A7[3][1] * f[4] + A7[3][2] * f[5] + A7[3][3] * f[6];
    double tau7 = fabs(is0 - is3);
    double alpha0 = C_W7[0] * (1.0 + PW(tau7 / (ss + is0)));
    double alpha1 = C_W7[1] * (1.0 + PW(tau7 / (ss + is1)));
    double alpha2 = C_W7[2] * (1.0 + PW(tau7 / (ss + is2)));
    double alpha3 = C_W7[3] * (1.0 + PW(tau7 / (ss + is3)));
    double alphaSum = alpha0 + alpha1 + alpha2 + alpha3;
    double omega0 = alpha0 / alphaSum;
    double omega1 = alpha1 / alphaSum;
    double omega2 = alpha2 / alphaSum;
    double omega3 = alpha3 / alphaSum;
    *alpha_sum = alphaSum;
    return omega0 * q40 + omega1 * q41 + omega2 * q42 + omega3 * q43;
}

/* hccs78's inner face (hccs78.cpp:81-139 for '+', :171-229 for '-'): the
 * WENO7-Z face blended with the 8-cell central value q8 (symmetric about the
 * face, the same expression for both signs) by theta = 1/(1 + (sum alpha -
 * 1)^2): (1 - theta) W7 + theta q8.  g: the upwind-oriented 7-cell WENO7
 * stencil; c[0..7]: cells m-4..m+3 around face m. */
static double hccs78_face(const double g[7], const double c[8]) {
    const double q8 = (-3.0 * (c[7] + c[0]) + 29.0 * (c[6] + c[1]) - 139.0 * (c[5] + c[2]) +
                       533.0 * (c[4] + c[3])) / 840.0;
    double alphaSum;
    const double w7 = weno7z_face_sum(g, &alphaSum);
    const double theta = 1.0 / (1.0 + PW(alphaSum - 1.0));
    return (1.0 - theta) * w7 + theta * q8;
}

/* One row of hccs77 (hccs77.cpp:79-162 for '+', :246-305 for '-').  g[0..6]:
 * the upwind-oriented 7-cell stencil of the row's cell i ('+': cells
 * i-3..i+3; '-': cells i+4..i-2).  WENO7-Z weights and candidates, the
 * 7th-order upwind compact value q7, theta = 1/(1 + (sum alpha - 1)^2);
 * theta > 1/2 gives the linear upwind compact row (2/7, 4/7, 1/7 | q7),
 * otherwise (2/7 theta, 1 - 3/7 theta, 1/7 theta | (1 - theta) W7 + theta q7).
 * Returns the upwind-side coupling lo, the diagonal b, the downwind-side
 * coupling hi and d. */
static void hccs77_row(const double g[7], double *lo, double *b, double *hi, double *d) {
    const double q7 = (-g[1] + 19.0 * g[2] + 239.0 * g[3] + 159.0 * g[4] + 4.0 * g[5]) / 420.0;
    double alphaSum;
    const double w7 = weno7z_face_sum(g, &alphaSum);
    const double theta = 1.0 / (1.0 + PW(alphaSum - 1.0));
    if (theta > 0.5) {
        *lo = 2.0 / 7.0;
        *b = 4.0 / 7.0;
        *hi = 1.0 / 7.0;
        *d = q7;
    } else {
        *lo = C_UPC[0] * theta;
        *b = 1.0 + (C_UPC[1] - 1.0) * theta;
        *hi = C_UPC[2] * theta;
        *d = w7 * (1.0 - theta) + q7 * theta;
    }
}

/* buffer (halo) width of a scheme (fieldOperator.cpp:128-175) */
static int halo_of(int scheme) {
    if (scheme == OR_WENO3JS) return 2;
    if (scheme == OR_UPWIND1) return 1;
    return scheme >= OR_WENO7 ? 4 : 3;
}

/* One compact-WENO row (crweno5.cpp:131-162 for '+', :311-341 for '-').
 * f[0..4] is the upwind-oriented 5-cell stencil of the row's cell i
 * ('+': cells i-2..i+2; '-': cells i+3..i-1), so f[1], f[2], f[3] are the
 * row's three right-hand-side cells in upwind order.  Returns the coefficient
 * of the upwind-side neighbour face (lo), the diagonal (b), the downwind-side
 * neighbour (hi) and the right-hand side d. */
static void crweno5_row(const double f[5], double *lo, double *b, double *hi, double *d) {
    const double ss = 1.0e-6;
    double is0 = G0 * SQ(f[0] - 2.0 * f[1] + f[2]) + G1 * SQ(f[0] - 4.0 * f[1] + 3.0 * f[2]);
    double is1 = G0 * SQ(f[1] - 2.0 * f[2] + f[3]) + G1 * SQ(f[1] - f[3]);
    double is2 = G0 * SQ(f[2] - 2.0 * f[3] + f[4]) + G1 * SQ(3.0 * f[2] - 4.0 * f[3] + f[4]);
    double alpha0 = C_CR5[0] / PW(ss + is0);
    double alpha1 = C_CR5[1] / PW(ss + is1);
    double alpha2 = C_CR5[2] / PW(ss + is2);
    double alphaSum = alpha0 + alpha1 + alpha2;
    double omega0 = alpha0 / alphaSum;
    double omega1 = alpha1 / alphaSum;
    double omega2 = alpha2 / alphaSum;
    *lo = 2.0 / 3.0 * omega0 + 1.0 / 3.0 * omega1;
    *b = 1.0 / 3.0 * omega0 + 2.0 / 3.0 * (omega1 + omega2);
    *hi = 1.0 / 3.0 * omega2;
    *d = 1.0 / 6.0 * omega0 * f[1] + (5.0 * (omega0 + omega1) + omega2) * f[2] / 6.0 +
         (omega1 + 5.0 * omega2) * f[3] / 6.0;
}

/* Gather the upwind-oriented stencil of face m from a line whose cell c lives
 * at line[c] (line must cover cells -3..n+2).  '+': cells m-3..m+1 (face m is
 * the left face of cell m, weno5js.cpp:108 writes face i+1 from cells
 * i-2..i+2); '-': cells m+2..m-2. */
static void face_stencil(const double *line, int m, int upwind, double f[5]) {
    for (int k = 0; k < 5; ++k) f[k] = upwind > 0 ? line[m - 3 + k] : line[m + 2 - k];
}

/* Thomas sweep exactly as crweno5.cpp:208-219: rows 0..M-1 with a (sub),
 * b (diag), c (super); row 0 must be an identity row.  Solution to x. */
static void thomas_ref(int M, double *a, double *b, double *c, double *d, double *x) {
    for (int i = 1; i < M; i++) {
        c[i] = c[i] / (b[i] - c[i - 1] * a[i]);
        d[i] = (d[i] - d[i - 1] * a[i]) / (b[i] - c[i - 1] * a[i]);
    }
    x[M - 1] = d[M - 1];
    for (int i = M - 2; i >= 0; i--) x[i] = d[i] - c[i] * x[i + 1];
}


/* One hybrid compact row of hccs (hccs.cpp:138-185 for '+', :375-420 for
 * '-').  f[0..4] is the upwind-oriented 5-cell stencil of the row's cell i
 * ('+': cells i-2..i+2; '-': cells i+3..i-1).  Returns the upwind-side
 * coupling lo, the diagonal b, the downwind-side coupling hi and d:
 *   WENO5-Z type weights with the CRWENO5 linear weights, eps = 1e-40,
 *   theta = 1/(1 + (sum alpha - 1)^2); theta > 1/2 takes the linear upwind
 *   compact row (2/7, 4/7, 1/7 | q7), otherwise the CRWENO5 row scaled by
 *   (1 - theta)/theta plus the linear one.  Squares are std::pow(x, 2) with a
 *   literal exponent in the reference, i.e. x*x. */
static void hccs_row(const double f[5], double *lo, double *b, double *hi, double *d) {
    const double ss = 1.0e-40;
    double is0 = G0 * SQ(f[0] - 2.0 * f[1] + f[2]) + G1 * SQ(f[0] - 4.0 * f[1] + 3.0 * f[2]);
    double is1 = G0 * SQ(f[1] - 2.0 * f[2] + f[3]) + G1 * SQ(f[1] - f[3]);
    double is2 = G0 * SQ(f[2] - 2.0 * f[3] + f[4]) + G1 * SQ(3.0 * f[2] - 4.0 * f[3] + f[4]);
    double q7 = (-f[0] + 19.0 * f[1] + 239.0 * f[2] + 159.0 * f[3] + 4.0 * f[4]) / 420.0;
    double tau = fabs(is2 - is0);
    double alpha0 = C_CR5[0] * (1.0 + SQ(tau / (is0 + ss)));
    double alpha1 = C_CR5[1] * (1.0 + SQ(tau / (is1 + ss)));
    double alpha2 = C_CR5[2] * (1.0 + SQ(tau / (is2 + ss)));
    double alphaSum = alpha0 + alpha1 + alpha2;
    double omega0 = alpha0 / alphaSum;
    double omega1 = alpha1 / alphaSum;
    double omega2 = alpha2 / alphaSum;
    double theta = 1.0 / (1.0 + SQ(alphaSum - 1.0));
    if (theta > 0.5) {
        *lo = 2.0 / 7.0;
        *b = 4.0 / 7.0;
        *hi = 1.0 / 7.0;
        *d = q7;
    } else {
        *lo = (2.0 / 3.0 * omega0 + 1.0 / 3.0 * omega1) * (1.0 - theta) / theta + C_UPC[0];
        *b = (1.0 / 3.0 * omega0 + 2.0 / 3.0 * (omega1 + omega2)) * (1.0 - theta) / theta + C_UPC[1];
        *hi = (1.0 / 3.0 * omega2) * (1.0 - theta) / theta + C_UPC[2];
        *d = (1.0 / 6.0 * omega0 * f[1] + (5.0 * (omega0 + omega1) + omega2) * f[2] / 6.0 +
              (omega1 + 5.0 * omega2) * f[3] / 6.0) *
                 (1.0 - theta) / theta +
             q7;
    }
}

/* Reconstruct all n+1 faces of one line.  line[] covers cells -3..n+2 (index
 * with line[c], c may be negative).  out[m], m=0..n.  This is what
 * interpolationInner + interpolationBoundaryL + interpolationBoundaryR
 * produce for one line (fieldOperator.cpp:387-465):
 *   faces 0..2   boundary-L form (halo), faces n-2..n boundary-R form,
 *   faces 3..n-3 inner form (for CRWENO5: the tridiagonal solve whose first
 *                and last rows are identity rows holding WENO5-JS values). */
static void reconstruct_line_ref(int scheme, int upwind, unsigned quirks, int n,
                                 const double *line, double *out, double *work) {
    double f[5];
    if (scheme == OR_WENO7) {
        /* face m: '+' cells m-4..m+2 (weno7js.cpp:123 writes face i+1 from
         * cells i-3..i+3), '-' cells m+3..m-3 */
        double g[7];
        for (int m = 0; m <= n; ++m) {
            for (int k = 0; k < 7; ++k) g[k] = upwind > 0 ? line[m - 4 + k] : line[m + 3 - k];
            out[m] = weno7_face(g);
        }
        return;
    }
    if (scheme == OR_HCCS) {
        /* hccs (hccs.cpp): faces 0..3 and n-3..n explicit WENO7 from the
         * halos (:538-980); the rows of cells i = 3..n-5 (faces 4..n-4,
         * :54-245 / :272-471) solved by the Thomas sweep (:232-245), the
         * first and last rows identity rows holding WENO7 values.  Every
         * WENO7 face here uses hccs's eps = 1e-40, not weno7js's 1e-20. */
        double g[7];
        for (int m = 0; m <= n; ++m) {
            if (m >= 4 && m <= n - 4) continue;
            for (int k = 0; k < 7; ++k) g[k] = upwind > 0 ? line[m - 4 + k] : line[m + 3 - k];
            out[m] = weno7_face_eps(g, 1.0e-40, 1);
        }
        int ibeg = 3, iend = n - 4, M = iend - ibeg;
        if (M < 2) return;
        double *a = work, *b = work + M, *c = work + 2 * M, *d = work + 3 * M, *x = work + 4 * M;
        for (int r = 0; r < M; ++r) {
            int i = ibeg + r;
            if (r == 0 || r == M - 1) {
                for (int k = 0; k < 7; ++k)
                    g[k] = upwind > 0 ? line[i + 1 - 4 + k] : line[i + 1 + 3 - k];
                a[r] = 0.0;
                b[r] = 1.0;
                c[r] = 0.0;
                d[r] = weno7_face_eps(g, 1.0e-40, 1);
            } else {
                double lo, bb, hi, dd;
                if (upwind > 0) {
                    for (int k = 0; k < 5; ++k) f[k] = line[i - 2 + k];
                    hccs_row(f, &lo, &bb, &hi, &dd);
                    a[r] = lo;
                    c[r] = hi;
                } else {
                    for (int k = 0; k < 5; ++k) f[k] = line[i + 3 - k];
                    hccs_row(f, &lo, &bb, &hi, &dd);
                    c[r] = lo;
                    a[r] = hi;
                }
                b[r] = bb;
                d[r] = dd;
            }
        }
        thomas_ref(M, a, b, c, d, x);
        for (int r = 0; r < M; ++r) out[ibeg + 1 + r] = x[r];
        return;
    }
    if (scheme == OR_UPWIND1) {
        /* upwind1st.cpp:40-368: face m takes the upwind cell, m-1 ('+') or m
         * ('-') */
        for (int m = 0; m <= n; ++m) out[m] = upwind > 0 ? line[m - 1] : line[m];
        return;
    }
    if (scheme == OR_WENO3JS) {
        /* weno3js.cpp: face m from cells m-2, m-1, m ('+') or m+1, m, m-1 ('-') */
        double g[3];
        for (int m = 0; m <= n; ++m) {
            for (int k = 0; k < 3; ++k) g[k] = upwind > 0 ? line[m - 2 + k] : line[m + 1 - k];
            out[m] = weno3js_face(g);
        }
        return;
    }
    if (scheme == OR_HCCS78) {
        /* hccs78 (hccs78.cpp): explicit.  Faces 0..3 and n-3..n WENO7-Z from
         * the halos (:242-732); faces 4..n-4 (inner, :44-229) blended with
         * q8. */
        double g[7], c[8], sum;
        for (int m = 0; m <= n; ++m) {
            for (int k = 0; k < 7; ++k) g[k] = upwind > 0 ? line[m - 4 + k] : line[m + 3 - k];
            if (m >= 4 && m <= n - 4) {
                for (int k = 0; k < 8; ++k) c[k] = line[m - 4 + k];
                out[m] = hccs78_face(g, c);
            } else {
                out[m] = weno7z_face_sum(g, &sum);
            }
        }
        return;
    }
    if (scheme == OR_HCCS77) {
        /* hccs77 (hccs77.cpp): faces 0..3 and n-3..n WENO7-Z from the halos
         * (:330-818); the rows of cells i = 3..n-5 (faces 4..n-4, :44-305)
         * solved by its Thomas sweep (:165-175), the first and last rows
         * identity rows holding WENO7-Z values. */
        double g[7], sum;
        for (int m = 0; m <= n; ++m) {
            if (m >= 4 && m <= n - 4) continue;
            for (int k = 0; k < 7; ++k) g[k] = upwind > 0 ? line[m - 4 + k] : line[m + 3 - k];
            out[m] = weno7z_face_sum(g, &sum);
        }
        int ibeg = 3, iend = n - 4, M = iend - ibeg;
        if (M < 2) return;
        double *a = work, *b = work + M, *c = work + 2 * M, *d = work + 3 * M, *x = work + 4 * M;
        for (int r = 0; r < M; ++r) {
            int i = ibeg + r;
            /* the row's stencil: '+' cells i-3..i+3, '-' cells i+4..i-2 */
            for (int k = 0; k < 7; ++k) g[k] = upwind > 0 ? line[i - 3 + k] : line[i + 4 - k];
            if (r == 0 || r == M - 1) {
                a[r] = 0.0;
                b[r] = 1.0;
                c[r] = 0.0;
                d[r] = weno7z_face_sum(g, &sum);
            } else {
                double lo, bb, hi, dd;
                hccs77_row(g, &lo, &bb, &hi, &dd);
                if (upwind > 0) {
                    a[r] = lo;
                    c[r] = hi;
                } else {
                    c[r] = lo;  /* hccs77.cpp:282-291: '-' couples face i+2 upwind */
                    a[r] = hi;
                }
                b[r] = bb;
                d[r] = dd;
            }
        }
        thomas_ref(M, a, b, c, d, x);
        for (int r = 0; r < M; ++r) out[ibeg + 1 + r] = x[r];
        return;
    }
    if (scheme == OR_CRWENO5) {
        for (int m = 0; m <= 2 && m <= n; ++m) {
            face_stencil(line, m, upwind, f);
            out[m] = weno5js_face(f);
        }
        for (int m = n - 2; m <= n; ++m) {
            if (m < 0) continue;
            face_stencil(line, m, upwind, f);
            out[m] = weno5js_face(f);
        }
        /* rows for cells i = 2..n-4, i.e. faces 3..n-3 (crweno5.cpp:76-219) */
        int ibeg = 2, iend = n - 3, M = iend - ibeg;
        if (M < 2) return;
        double *a = work, *b = work + M, *c = work + 2 * M, *d = work + 3 * M, *x = work + 4 * M;
        for (int r = 0; r < M; ++r) {
            int i = ibeg + r;
            if (r == 0 || r == M - 1) {
                face_stencil(line, i + 1, upwind, f);
                a[r] = 0.0;
                b[r] = 1.0;
                c[r] = 0.0;
                d[r] = weno5js_face(f);
            } else {
                double lo, bb, hi, dd;
                if (upwind > 0) {
                    for (int k = 0; k < 5; ++k) f[k] = line[i - 2 + k];
                    crweno5_row(f, &lo, &bb, &hi, &dd);
                    a[r] = lo;  /* couples face i   (crweno5.cpp:156) */
                    c[r] = hi;  /* couples face i+2 (crweno5.cpp:158) */
                } else {
                    for (int k = 0; k < 5; ++k) f[k] = line[i + 3 - k];
                    crweno5_row(f, &lo, &bb, &hi, &dd);
                    c[r] = lo;  /* crweno5.cpp:335: upwind side is face i+2 */
                    a[r] = hi;  /* crweno5.cpp:337 */
                }
                b[r] = bb;
                d[r] = dd;
            }
        }
        thomas_ref(M, a, b, c, d, x);
        for (int r = 0; r < M; ++r) out[ibeg + 1 + r] = x[r];
        return;
    }
    for (int m = 0; m <= n; ++m) {
        face_stencil(line, m, upwind, f);
        int inner = (m >= 3 && m <= n - 3);
        if (scheme == OR_WENO5JS)
            out[m] = weno5js_face(f);
        else
            out[m] = weno5z_face(f, upwind > 0 && inner && (quirks & OR_Q_WENOZ_BETA2));
    }
}

/* Solve the periodic (cyclic) tridiagonal system a x[i-1] + b x[i] + c x[i+1]
 * = d, i = 0..n-1 with wrap-around, by Sherman-Morrison on two Thomas solves.
 * Used by the periodic CRWENO5 form (quirk bit OR_Q_CRWENO_BOUNDED cleared),
 * which the reference does not have. */
static void cyclic_solve(int n, const double *a, const double *b, const double *c,
                         const double *d, double *x, double *w) {
    double *bb = w, *u = w + n, *cp = w + 2 * n, *dp = w + 3 * n, *z = w + 4 * n;
    double gamma = -b[0];
    for (int i = 0; i < n; ++i) bb[i] = b[i];
    bb[0] = b[0] - gamma;
    bb[n - 1] = b[n - 1] - a[0] * c[n - 1] / gamma;
    /* Thomas on (a, bb, c) for rhs d -> x and rhs u -> z */
    for (int pass = 0; pass < 2; ++pass) {
        const double *rhs = d;
        double *sol = x;
        if (pass == 1) {
            for (int i = 0; i < n; ++i) u[i] = 0.0;
            u[0] = gamma;
            u[n - 1] = c[n - 1];
            rhs = u;
            sol = z;
        }
        cp[0] = c[0] / bb[0];
        dp[0] = rhs[0] / bb[0];
        for (int i = 1; i < n; ++i) {
            double den = bb[i] - a[i] * cp[i - 1];
            cp[i] = c[i] / den;
            dp[i] = (rhs[i] - a[i] * dp[i - 1]) / den;
        }
        sol[n - 1] = dp[n - 1];
        for (int i = n - 2; i >= 0; --i) sol[i] = dp[i] - cp[i] * sol[i + 1];
    }
    double fact = (x[0] + a[0] * x[n - 1] / gamma) / (1.0 + z[0] + a[0] * z[n - 1] / gamma);
    for (int i = 0; i < n; ++i) x[i] -= fact * z[i];
}

static void reconstruct_line_periodic_crweno(int upwind, int n, const double *line, double *out,
                                             double *work) {
    double *a = work, *b = work + n, *c = work + 2 * n, *d = work + 3 * n, *x = work + 4 * n;
    double *w = work + 5 * n;
    double f[5];
    for (int m = 0; m < n; ++m) {
        int i = m - 1; /* row of face m belongs to cell i = m-1 */
        double lo, bb, hi, dd;
        if (upwind > 0) {
            for (int k = 0; k < 5; ++k) f[k] = line[i - 2 + k];
            crweno5_row(f, &lo, &bb, &hi, &dd);
            a[m] = lo;
            c[m] = hi;
        } else {
            for (int k = 0; k < 5; ++k) f[k] = line[i + 3 - k];
            crweno5_row(f, &lo, &bb, &hi, &dd);
            c[m] = lo;
            a[m] = hi;
        }
        b[m] = bb;
        d[m] = dd;
    }
    cyclic_solve(n, a, b, c, d, x, w);
    for (int m = 0; m < n; ++m) out[m] = x[m];
    out[n] = x[0];
}

int or_reconstruct_field(int scheme, int upwind, unsigned quirks, int nx, int ny, int nz,
                         const double *in, const double *halo_l, const double *halo_r,
                         double *out) {
    if (nx < 5 || (upwind != 1 && upwind != -1)) return -1;
    const int H = halo_of(scheme);
    double *buf = (double *)malloc(sizeof(double) * (size_t)(nx + 2 * H));
    double *work = (double *)malloc(sizeof(double) * (size_t)(10 * (nx + 1)));
    double *line = buf + H;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
            for (int c = 0; c < H; ++c) {
                line[c - H] = halo_l[c + H * (j + ny * k)];
                line[nx + c] = halo_r[c + H * (j + ny * k)];
            }
            for (int i = 0; i < nx; ++i) line[i] = in[i + nx * (j + ny * k)];
            reconstruct_line_ref(scheme, upwind, quirks, nx, line,
                                 out + (size_t)(nx + 1) * (j + ny * k), work);
        }
    free(buf);
    free(work);
    return 0;
}

/* ------------------------------------------------------------------ CD6 --- */

/* centraldifference6th.cpp:44-46 (inner) and :111-113 / :179-181 (halo). */
static double cd6_at(const double *line, int i, double dx) {
    return (CD6[2] * (line[i + 3] - line[i - 3]) + CD6[1] * (line[i + 2] - line[i - 2]) +
            CD6[0] * (line[i + 1] - line[i - 1])) /
           dx;
}

/* centraldifference2nd.cpp:44 (inner), :82 / :136 (halo): one form everywhere. */
static double cd2_at(const double *line, int i, double dx) {
    return 0.5 * (line[i + 1] - line[i - 1]) / dx;
}

/* centraldifference8th.cpp:50-60 (inner cells): the two one-sided sums, then
 * their difference. */
static double cd8_inner_at(const double *line, int i, double dx) {
    const double an = CD8[3] * line[i - 4] + CD8[2] * line[i - 3] + CD8[1] * line[i - 2] +
                      CD8[0] * line[i - 1];
    const double ap = CD8[0] * line[i + 1] + CD8[1] * line[i + 2] + CD8[2] * line[i + 3] +
                      CD8[3] * line[i + 4];
    return (ap - an) / dx;
}

/* centraldifference8th.cpp:120-123 / :188-191 (cells within the tile width
 * of a line end): symmetric differences. */
static double cd8_edge_at(const double *line, int i, double dx) {
    return (CD8[3] * (line[i + 4] - line[i - 4]) + CD8[2] * (line[i + 3] - line[i - 3]) +
            CD8[1] * (line[i + 2] - line[i - 2]) + CD8[0] * (line[i + 1] - line[i - 1])) /
           dx;
}

/* derivative at cell i of an n-cell line whose halos are filled as far as the
 * scheme reaches; `tile` is the reference's tilesize (the inviscid scheme's
 * bufferSize, fieldOperator.cpp:520-610): cd8 cells within it of a line end
 * take the boundary form. */
static double cd_at(int scheme, int tile, const double *line, int n, int i, double dx) {
    if (scheme == OR_CD2) return cd2_at(line, i, dx);
    if (scheme == OR_CD8)
        return (i < tile || i >= n - tile) ? cd8_edge_at(line, i, dx) : cd8_inner_at(line, i, dx);
    return cd6_at(line, i, dx);
}

int or_cd_field(int scheme, int tile, int nx, int ny, int nz, double dx, const double *in,
                const double *halo_l, const double *halo_r, double *out) {
    const int reach = scheme == OR_CD2 ? 1 : (scheme == OR_CD8 ? 4 : 3);
    if (tile < 1 || tile > 4 || tile < reach || nx < 2 * tile) return -1;
    double *buf = (double *)malloc(sizeof(double) * (size_t)(nx + 2 * tile));
    double *line = buf + tile;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
            for (int c = 0; c < tile; ++c) {
                line[c - tile] = halo_l[c + tile * (j + ny * k)];
                line[nx + c] = halo_r[c + tile * (j + ny * k)];
            }
            for (int i = 0; i < nx; ++i) line[i] = in[i + nx * (j + ny * k)];
            for (int i = 0; i < nx; ++i)
                out[i + nx * (j + ny * k)] = cd_at(scheme, tile, line, nx, i, dx);
        }
    free(buf);
    return 0;
}

int or_cd6_field(int nx, int ny, int nz, double dx, const double *in, const double *halo_l,
                 const double *halo_r, double *out) {
    double *buf = (double *)malloc(sizeof(double) * (size_t)(nx + 6));
    double *line = buf + 3;
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j) {
            for (int c = 0; c < 3; ++c) {
                line[c - 3] = halo_l[c + 3 * (j + ny * k)];
                line[nx + c] = halo_r[c + 3 * (j + ny * k)];
            }
            for (int i = 0; i < nx; ++i) line[i] = in[i + nx * (j + ny * k)];
            for (int i = 0; i < nx; ++i) out[i + nx * (j + ny * k)] = cd6_at(line, i, dx);
        }
    free(buf);
    return 0;
}

/* ------------------------------------------------------------ physics ---- */

typedef struct {
    const or_box *b;
    const double *const *q;
    double *const *prim;
} c2p_ctx;

static void c2p_range(void *vc, int part, long lo, long hi) {
    /* physicsModel.cpp:317-356 */
    const c2p_ctx *x = (const c2p_ctx *)vc;
    const or_box *b = x->b;
    const double *const *q = x->q;
    double *const *prim = x->prim;
    const double gamma = b->gamma, Mach = b->mach;
    (void)part;
    for (long n = lo; n < hi; ++n) {
        double rho = q[0][n];
        double u = q[1][n] / rho;
        double v = q[2][n] / rho;
        double w = q[3][n] / rho;
        double E = q[4][n];
        double p = (E - 0.5 * rho * (u * u + v * v + w * w)) * (gamma - 1.0);
        if (b->quirks & OR_Q_FABS_PRESSURE) p = fabs(p);
        double e = p / rho / (gamma - 1.0);
        double alpha = sqrt(gamma * p / rho);
        double T = gamma * Mach * Mach * p / rho;
        prim[0][n] = rho;
        prim[1][n] = u;
        prim[2][n] = v;
        prim[3][n] = w;
        prim[4][n] = p;
        prim[5][n] = T;
        prim[6][n] = e;
        prim[7][n] = alpha;
    }
}

void or_con2prim(const or_box *b, const double *const q[5], double *const prim[8]) {
    const long N = (long)b->nx * b->ny * b->nz;
    c2p_ctx x = {b, q, prim};
    or_parallel(N, c2p_range, &x);
}

typedef struct {
    const or_box *b;
    const double *const *q;
    const double *const *prim;
    double *const *fl, *const *fr;
    int d;
    double mpart[OR_MAX_THREADS];
} split_ctx;

static void lf_range(void *vc, int part, long lo, long hi) {
    split_ctx *x = (split_ctx *)vc;
    const int d = x->d;
    const double *const *q = x->q;
    const double *const *prim = x->prim;
    double m = x->mpart[part];
    for (long n = lo; n < hi; ++n) {
        double un = prim[1 + d][n];
        double p0 = prim[4][n];
        double alpha0 = prim[7][n];
        double Q[5] = {q[0][n], q[1][n], q[2][n], q[3][n], q[4][n]};
        double lam = fabs(un) + alpha0;
        m = fmax(lam, m);
        double flux[5];
        flux[0] = un * Q[0];
        flux[1] = un * Q[1];
        flux[2] = un * Q[2];
        flux[3] = un * Q[3];
        flux[1 + d] = un * Q[1 + d] + p0;
        flux[4] = un * (Q[4] + p0);
        for (int e = 0; e < 5; ++e) {
            x->fl[e][n] = 0.5 * (flux[e] + lam * Q[e]);
            x->fr[e][n] = 0.5 * (flux[e] - lam * Q[e]);
        }
    }
    x->mpart[part] = m;
}

/* one direction of a split over all cells; the running maximum `run` is
 * continued part by part with fmax */
static double split_direction(split_ctx *x, or_range_fn fn, long N, double run) {
    for (int i = 0; i < OR_MAX_THREADS; ++i) x->mpart[i] = run;
    int T = or_parallel(N, fn, x);
    for (int i = 0; i < T; ++i) run = fmax(x->mpart[i], run);
    return run;
}

void or_lf_split(const or_box *b, const double *const q[5], const double *const prim[8],
                 double *const fl[3][5], double *const fr[3][5], double eig[3]) {
    /* physicsModel.cpp:520-679.  The three loops run in the reference's order
     * (xi, eta, zeta) so the running fmax values match. */
    const long N = (long)b->nx * b->ny * b->nz;
    double me[3] = {0.0, 0.0, 0.0};
    split_ctx x;
    x.b = b;
    x.q = q;
    x.prim = prim;
    for (int d = 0; d < 3; ++d) {
        int slot = d;
        if (d == 2 && (b->quirks & OR_Q_ZETA_EIGEN)) slot = 1; /* :653-654 */
        x.fl = fl[d];
        x.fr = fr[d];
        x.d = d;
        me[slot] = split_direction(&x, lf_range, N, me[slot]);
    }
    eig[0] = me[0];
    eig[1] = me[1];
    eig[2] = me[2];
}

/* physicsModel.cpp:1181-1278: the Mach-number and pressure splittings.
 * AUSM squares with pow(x, 2) (an int exponent, promoted) and AUSMp with
 * pow(x, 2.0): the same libm call. */
static double ausm_mach_l(double mach) {
    if (fabs(mach) < 1.0) return 0.25 * pow(mach + 1.0, 2.0) + 0.125 * pow(mach * mach - 1, 2.0);
    return 0.50 * (mach + fabs(mach));
}
static double ausm_mach_r(double mach) {
    if (fabs(mach) < 1.0) return -0.25 * pow(mach - 1.0, 2.0) - 0.125 * pow(mach * mach - 1, 2.0);
    return 0.50 * (mach - fabs(mach));
}
static double ausm_p_l(double mach, double p) {
    if (fabs(mach) < 1.0) return p * (mach + 1.0) / 2.0;
    return 0.50 * p * (mach + fabs(mach)) / mach;
}
static double ausm_p_r(double mach, double p) {
    if (fabs(mach) < 1.0) return -p * (mach - 1.0) / 2.0;
    return 0.5 * p * (mach - fabs(mach)) / mach;
}
static double ausmp_p_l(double mach, double p) {
    if (fabs(mach) < 1.0)
        return p * (0.25 * pow(mach + 1.0, 2.0) * (2.0 - mach) +
                    0.1875 * mach * pow(mach * mach - 1.0, 2.0));
    return 0.50 * p * (mach + fabs(mach)) / mach;
}
static double ausmp_p_r(double mach, double p) {
    if (fabs(mach) < 1.0)
        return p * (0.25 * pow(mach - 1.0, 2.0) * (2.0 + mach) -
                    0.1875 * mach * pow(mach * mach - 1.0, 2.0));
    return 0.5 * p * (mach - fabs(mach)) / mach;
}

static void ausm_range(void *vc, int part, long lo, long hi) {
    split_ctx *x = (split_ctx *)vc;
    const int d = x->d;
    const int plus = x->b->riemann == OR_AUSMP;
    const double *const *q = x->q;
    const double *const *prim = x->prim;
    double *const *fl = x->fl, *const *fr = x->fr;
    double m = x->mpart[part];
    for (long n = lo; n < hi; ++n) {
        double un = prim[1 + d][n];
        double p0 = prim[4][n];
        double alpha0 = prim[7][n];
        double mach = un / alpha0;
        double machp = ausm_mach_l(mach);
        double machn = ausm_mach_r(mach);
        double p_p = plus ? ausmp_p_l(mach, p0) : ausm_p_l(mach, p0);
        double p_n = plus ? ausmp_p_r(mach, p0) : ausm_p_r(mach, p0);
        m = fmax(fabs(un) + alpha0, m);
        for (int e = 0; e < 4; ++e) {
            fl[e][n] = machp * alpha0 * q[e][n];
            fr[e][n] = machn * alpha0 * q[e][n];
        }
        fl[1 + d][n] = machp * alpha0 * q[1 + d][n] + p_p;
        fr[1 + d][n] = machn * alpha0 * q[1 + d][n] + p_n;
        fl[4][n] = machp * alpha0 * q[4][n] + machp * alpha0 * p0;
        fr[4][n] = machn * alpha0 * q[4][n] + machn * alpha0 * p0;
    }
    x->mpart[part] = m;
}

void or_ausm_split(const or_box *b, const double *const q[5], const double *const prim[8],
                   double *const fl[3][5], double *const fr[3][5], double eig[3]) {
    /* physicsModel.cpp:777-929 (AUSM), :1027-1178 (AUSMp): directions in the
     * reference's order; (machp*alpha0)*Q evaluated left to right. */
    const long N = (long)b->nx * b->ny * b->nz;
    double me[3] = {0.0, 0.0, 0.0};
    split_ctx x;
    x.b = b;
    x.q = q;
    x.prim = prim;
    for (int d = 0; d < 3; ++d) {
        x.fl = fl[d];
        x.fr = fr[d];
        x.d = d;
        me[d] = split_direction(&x, ausm_range, N, me[d]);
    }
    eig[0] = me[0];
    eig[1] = me[1];
    eig[2] = me[2];
}

/* physicsModel.cpp:193-266 (+ an extra power-law model). */
static void viscosity(const or_box *b, double T, double *miu, double *coeff) {
    double m;
    if (b->visc_model == OR_SUTHERLAND) {
        double non_dim_T_ref = b->t_ref / b->t_inf;
        m = (1.0 + non_dim_T_ref) / (T + non_dim_T_ref) * pow(T, 1.5) / b->reynolds;
    } else if (b->visc_model == OR_CONSTANT) {
        m = 1.0 / b->reynolds;
    } else {
        m = pow(T, b->powerlaw_exp) / b->reynolds;
    }
    *miu = m;
    *coeff = m / ((b->gamma - 1.0) * b->mach * b->mach * b->prandtl);
}

/* --------------------------------------------------------------- RHS ---- */

typedef struct {
    long base;
    long stride;
} line_t;

static long dir_stride(const or_box *b, int d) {
    return d == 0 ? 1 : (d == 1 ? (long)b->nx : (long)b->nx * b->ny);
}
static int dir_len(const or_box *b, int d) { return d == 0 ? b->nx : (d == 1 ? b->ny : b->nz); }

/* enumerate line bases for direction d */
static long line_base(const or_box *b, int d, int a, int c) {
    /* a, c: the two transverse indices in increasing memory order */
    if (d == 0) return (long)b->nx * (a + (long)b->ny * c);  /* a=j, c=k */
    if (d == 1) return a + (long)b->nx * b->ny * c;          /* a=i, c=k */
    return a + (long)b->nx * c;                              /* a=i, c=j */
}
static void line_counts(const or_box *b, int d, int *na, int *nc) {
    if (d == 0) { *na = b->ny; *nc = b->nz; }
    else if (d == 1) { *na = b->nx; *nc = b->nz; }
    else { *na = b->nx; *nc = b->ny; }
}

static void gather_periodic(const double *src, long base, long stride, int n, double *line) {
    for (int c = -4; c < n + 4; ++c) {
        int cc = ((c % n) + n) % n;
        line[c] = src[base + (long)cc * stride];
    }
}

typedef struct {
    const or_box *b;
    int d, n, na, nc, periodic_cr;
    long s;
    double delta;
    double *const *fl, *const *fr, *const *df;
} inv_ctx;

/* lines lo..hi-1 of the 5 * nc * na (equation, c, a) lines of a direction */
static void inv_range(void *vc, int part, long lo, long hi) {
    const inv_ctx *x = (const inv_ctx *)vc;
    const or_box *b = x->b;
    const int d = x->d, n = x->n;
    const long s = x->s;
    (void)part;
    double *buf = (double *)malloc(sizeof(double) * (size_t)(n + 8));
    double *line = buf + 4;
    double *rp = (double *)malloc(sizeof(double) * (size_t)(n + 1));
    double *rn = (double *)malloc(sizeof(double) * (size_t)(n + 1));
    double *work = (double *)malloc(sizeof(double) * (size_t)(10 * (n + 1)));
    const long per_e = (long)x->nc * x->na;
    for (long L = lo; L < hi; ++L) {
        const int e = (int)(L / per_e);
        const long r = L - e * per_e;
        const int c = (int)(r / x->na), a = (int)(r - (long)c * x->na);
        long base = line_base(b, d, a, c);
        gather_periodic(x->fl[e], base, s, n, line);
        if (x->periodic_cr)
            reconstruct_line_periodic_crweno(1, n, line, rp, work);
        else
            reconstruct_line_ref(b->scheme[d], 1, b->quirks, n, line, rp, work);
        gather_periodic(x->fr[e], base, s, n, line);
        if (x->periodic_cr)
            reconstruct_line_periodic_crweno(-1, n, line, rn, work);
        else
            reconstruct_line_ref(b->scheme[d], -1, b->quirks, n, line, rn, work);
        for (int m = 0; m <= n; ++m) rp[m] = rp[m] + rn[m];
        for (int i = 1; i <= n; ++i) {
            double df_loc = rp[i] - rp[i - 1];
            x->df[e][base + (long)(i - 1) * s] = df_loc / x->delta;
        }
    }
    free(buf);
    free(rp);
    free(rn);
    free(work);
}

/* Inviscid derivative of one direction (euler3d.cpp:307-387 solveInv,
 * :23-56 combineFluxLR, :143-253 setDerivatives*Inv): for every equation,
 * F^ = F^+(face) + F^-(face), dF/dx(cell i) = (F^[i+1] - F^[i]) / delta. */
static void inviscid_direction(const or_box *b, int d, double *const fl[5], double *const fr[5],
                               double *const df[5]) {
    inv_ctx x;
    x.b = b;
    x.d = d;
    x.n = dir_len(b, d);
    x.s = dir_stride(b, d);
    x.delta = d == 0 ? b->dx : (d == 1 ? b->dy : b->dz);
    line_counts(b, d, &x.na, &x.nc);
    x.periodic_cr = b->scheme[d] == OR_CRWENO5 && !(b->quirks & OR_Q_CRWENO_BOUNDED);
    x.fl = fl;
    x.fr = fr;
    x.df = df;
    or_parallel(5L * x.nc * x.na, inv_range, &x);
}

typedef struct {
    const or_box *b;
    int d, n, na, scheme, tile;
    long s;
    double delta;
    const double *src;
    double *dst;
} cd6_ctx;

static void cd6_range(void *vc, int part, long lo, long hi) {
    const cd6_ctx *x = (const cd6_ctx *)vc;
    const int n = x->n;
    (void)part;
    double *buf = (double *)malloc(sizeof(double) * (size_t)(n + 8));
    double *line = buf + 4;
    for (long L = lo; L < hi; ++L) {
        const int c = (int)(L / x->na), a = (int)(L - (long)c * x->na);
        long base = line_base(x->b, x->d, a, c);
        gather_periodic(x->src, base, x->s, n, line);
        for (int i = 0; i < n; ++i)
            x->dst[base + (long)i * x->s] = cd_at(x->scheme, x->tile, line, n, i, x->delta);
    }
    free(buf);
}

/* The direction's differential scheme along direction d of a periodic field
 * (the halo exchange with one rank is the periodic wrap), with the tilesize
 * the reference passes it: the inviscid scheme's bufferSize.  With cd8 and a
 * bufferSize below 4 the reference's stencils read outside their halo buffers
 * and across line starts (centraldifference8th.cpp:46-57, :101-113); here
 * they read the periodic neighbours. */
static void cd_direction(const or_box *b, int d, const double *src, double *dst) {
    cd6_ctx x;
    int nc;
    x.b = b;
    x.d = d;
    x.scheme = b->vis[d];
    x.tile = halo_of(b->scheme[d]);
    x.n = dir_len(b, d);
    x.s = dir_stride(b, d);
    x.delta = d == 0 ? b->dx : (d == 1 ? b->dy : b->dz);
    line_counts(b, d, &x.na, &nc);
    x.src = src;
    x.dst = dst;
    or_parallel((long)nc * x.na, cd6_range, &x);
}

static double *alloc_fields(int count, long N, double **ptrs) {
    double *blk = (double *)calloc((size_t)count * (size_t)N, sizeof(double));
    for (int i = 0; i < count; ++i) ptrs[i] = blk + (size_t)i * N;
    return blk;
}

typedef struct {
    const or_box *b;
    const double *const *g;
    const double *const *prim;
    double *const *fv;
} visc_ctx;

/* solveViscousFlux (NaiverStokes3d.cpp:177-303) for cells lo..hi-1 */
static void visc_range(void *vc, int part, long lo, long hi) {
    const visc_ctx *x = (const visc_ctx *)vc;
    const or_box *b = x->b;
    const double *const *g = x->g;
    const double *const *prim = x->prim;
    double *const *fv = x->fv;
    const double c23 = 2.0 / 3.0;
    int offdiag = (b->quirks & OR_Q_OFFDIAG_DIV) != 0;
    (void)part;
    for (long n = lo; n < hi; ++n) {
        double ux = g[0][n], uy = g[1][n], uz = g[2][n];
        double vx = g[3][n], vy = g[4][n], vz = g[5][n];
        double wx = g[6][n], wy = g[7][n], wz = g[8][n];
        double tx = g[9][n], ty = g[10][n], tz = g[11][n];
        double grad = ux + vy + wz;
        double miu0, coeff0;
        viscosity(b, prim[5][n], &miu0, &coeff0);
        double tau_xx = miu0 * (2.0 * ux - c23 * grad);
        double tau_xy = offdiag ? miu0 * (uy + vx - c23 * grad) : miu0 * (uy + vx);
        double tau_xz = offdiag ? miu0 * (uz + wx - c23 * grad) : miu0 * (uz + wx);
        double tau_yy = miu0 * (2.0 * vy - c23 * grad);
        double tau_yz = offdiag ? miu0 * (vz + wy - c23 * grad) : miu0 * (vz + wy);
        double tau_zz = miu0 * (2.0 * wz - c23 * grad);
        double tau_tx = coeff0 * tx, tau_ty = coeff0 * ty, tau_tz = coeff0 * tz;
        double u = prim[1][n], v = prim[2][n], w = prim[3][n];
        fv[0][n] = 0.0;
        fv[1][n] = tau_xx;
        fv[2][n] = tau_xy;
        fv[3][n] = tau_xz;
        fv[4][n] = u * tau_xx + v * tau_xy + w * tau_xz + tau_tx;
        fv[5][n] = 0.0;
        fv[6][n] = tau_xy;
        fv[7][n] = tau_yy;
        fv[8][n] = tau_yz;
        fv[9][n] = u * tau_xy + v * tau_yy + w * tau_yz + tau_ty;
        fv[10][n] = 0.0;
        fv[11][n] = tau_xz;
        fv[12][n] = tau_yz;
        fv[13][n] = tau_zz;
        fv[14][n] = u * tau_xz + v * tau_yz + w * tau_zz + tau_tz;
    }
}

typedef struct {
    int navier_stokes;
    double *const *dinv, *const *dvis, *const *rhs;
} sum_ctx;

/* solveRHS (NaiverStokes3d.cpp:385-499 / euler3d.cpp:389-457) for cells
 * lo..hi-1, in the reference's summation order */
static void sum_range(void *vc, int part, long lo, long hi) {
    const sum_ctx *x = (const sum_ctx *)vc;
    (void)part;
    for (int e = 0; e < 5; ++e)
        for (long n = lo; n < hi; ++n) {
            double r = x->dinv[e][n];
            r += x->dinv[5 + e][n];
            r += x->dinv[10 + e][n];
            if (x->navier_stokes) {
                r -= x->dvis[e][n];
                r -= x->dvis[5 + e][n];
                r -= x->dvis[10 + e][n];
            }
            x->rhs[e][n] = r;
        }
}

double or_rhs(const or_box *b, const double *const q[5], double *const rhs[5]) {
    const long N = (long)b->nx * b->ny * b->nz;
    double *prim[8], *flp[15], *frp[15], *dinv[15];
    double *blk_prim = alloc_fields(8, N, prim);
    double *blk_fl = alloc_fields(15, N, flp);
    double *blk_fr = alloc_fields(15, N, frp);
    double *blk_d = alloc_fields(15, N, dinv);
    double *fl[3][5], *fr[3][5];
    for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 5; ++e) {
            fl[d][e] = flp[d * 5 + e];
            fr[d][e] = frp[d * 5 + e];
        }
    double eig[3];
    or_con2prim(b, q, prim);                 /* NaiverStokes3d.cpp:46 */
    if (b->riemann == OR_LF) /* :48, physicsModel::solveRiemann */
        or_lf_split(b, q, (const double *const *)prim, fl, fr, eig);
    else
        or_ausm_split(b, q, (const double *const *)prim, fl, fr, eig);
    for (int d = 0; d < 3; ++d) inviscid_direction(b, d, fl[d], fr[d], dinv + 5 * d); /* :52 */
    free(blk_fl); /* the split fluxes are not needed again */
    free(blk_fr);
    blk_fl = blk_fr = NULL;

    double *dvis[15] = {0};
    double *blk_v = NULL;
    if (b->navier_stokes) {
        /* solveGrads (NaiverStokes3d.cpp:87-175): derivatives of u, v, w, T
         * along x, y, z with each direction's differential scheme */
        double *g[12];
        double *blk_g = alloc_fields(12, N, g);
        const double *src[4] = {prim[1], prim[2], prim[3], prim[5]};
        for (int vix = 0; vix < 4; ++vix)
            for (int d = 0; d < 3; ++d) cd_direction(b, d, src[vix], g[vix * 3 + d]);
        /* solveViscousFlux (NaiverStokes3d.cpp:177-303) */
        double *fv[15];
        double *blk_fv = alloc_fields(15, N, fv);
        visc_ctx vx_ = {b, (const double *const *)g, (const double *const *)prim, fv};
        or_parallel(N, visc_range, &vx_);
        free(blk_g);
        /* setDerivativesVis (NaiverStokes3d.cpp:305-369) */
        blk_v = alloc_fields(15, N, dvis);
        for (int d = 0; d < 3; ++d)
            for (int e = 0; e < 5; ++e) cd_direction(b, d, fv[d * 5 + e], dvis[d * 5 + e]);
        free(blk_fv);
    }
    /* solveRHS: NaiverStokes3d.cpp:385-499 / euler3d.cpp:389-457 */
    sum_ctx sx = {b->navier_stokes, dinv, dvis, rhs};
    or_parallel(N, sum_range, &sx);
    free(blk_prim);
    free(blk_fl);
    free(blk_fr);
    free(blk_d);
    free(blk_v);
    /* getDt (euler3d.cpp:459-466) */
    double dt_xi = b->dx / eig[0];
    double dt_eta = b->dy / eig[1];
    double dt_zeta = b->dz / eig[2];
    return 1.0 / (1.0 / dt_xi + 1.0 / dt_eta + 1.0 / dt_zeta);
}

/* ------------------------------------------------------------- RK3 ------- */

typedef struct {
    int stage;
    double dt;
    const double *const *rhs, *const *un;
    double *const *ui;
} rk_ctx;

static void rk_range(void *vc, int part, long lo, long hi) {
    /* TVD-RK3.h:9-12 coefficients; TVD-RK3.cpp:76-196 */
    static const double c[3][2] = {{1.0, 1.0}, {3.0 / 4.0, 1.0 / 4.0}, {1.0 / 3.0, 2.0 / 3.0}};
    const rk_ctx *x = (const rk_ctx *)vc;
    const int stage = x->stage;
    const double dt = x->dt;
    (void)part;
    for (int e = 0; e < 5; ++e)
        for (long i = lo; i < hi; ++i) {
            double r = -x->rhs[e][i];
            if (stage == 0) {
                double u = x->ui[e][i];
                x->ui[e][i] = c[0][0] * u + c[0][1] * r * dt;
            } else {
                double u = x->un[e][i];
                double uk = x->ui[e][i];
                x->ui[e][i] = c[stage][0] * u + c[stage][1] * (r * dt + uk);
            }
        }
}

void or_rk3_stage(int stage, long n, double dt, const double *const rhs[5],
                  const double *const un[5], double *const ui[5]) {
    rk_ctx x = {stage, dt, rhs, un, ui};
    or_parallel(n, rk_range, &x);
}

void or_run_steps(const or_box *b, double cfl, int nsteps, double *const q[5], double *dt,
                  double *res) {
    const long N = (long)b->nx * b->ny * b->nz;
    double *un[5], *rhs[5];
    double *blk_un = alloc_fields(5, N, un);
    double *blk_r = alloc_fields(5, N, rhs);
    for (int s = 0; s < nsteps; ++s) {
        double dt_global = 0.0;
        for (int stage = 0; stage < 3; ++stage) {
            double dt_local = or_rhs(b, (const double *const *)q, rhs);
            if (stage == 0) { /* PDEData3d.cpp:161-165 */
                for (int e = 0; e < 5; ++e) memcpy(un[e], q[e], sizeof(double) * (size_t)N);
                dt_global = dt_local * cfl;
            }
            or_rk3_stage(stage, N, dt_global, (const double *const *)rhs,
                         (const double *const *)un, q);
        }
        /* setRES (PDEData3d.cpp:178-213) */
        double res_this = 0.0;
        for (int e = 0; e < 5; ++e)
            for (long i = 0; i < N; ++i) res_this += SQ(q[e][i] - un[e][i]);
        dt[s] = dt_global;
        res[s] = sqrt(res_this / (double)((size_t)N * 5u)) / dt_global;
    }
    free(blk_un);
    free(blk_r);
}

/* ------------------------------------------------------------- ICs ------- */

void or_init_tgv(const or_box *b, double x0, double y0, double z0, double *const q[5]) {
    /* mesh centres block.cpp:120-122 with one rank (coord 0); TGV :369-394 */
    const double gamma = b->gamma, mach = b->mach;
    for (int k = 0; k < b->nz; k++)
        for (int j = 0; j < b->ny; j++)
            for (int i = 0; i < b->nx; i++) {
                long idx = i + (long)b->nx * (j + (long)b->ny * k);
                double xc = 0.0 + b->dx * (0.5 + i) - x0;
                double yc = 0.0 + b->dy * (0.5 + j) - y0;
                double zc = 0.0 + b->dz * (0.5 + k) - z0;
                double rho0 = 1.0;
                double u0 = sin(xc) * cos(yc) * cos(zc);
                double v0 = -cos(xc) * sin(yc) * cos(zc);
                double w0 = 0.0;
                double p0 = 1.0 / (gamma * mach * mach) +
                            ((cos(2.0 * zc) + 2.0) * (cos(2.0 * xc) + cos(2.0 * yc)) - 2.0) / 16.0;
                q[0][idx] = rho0;
                q[1][idx] = rho0 * u0;
                q[2][idx] = rho0 * v0;
                q[3][idx] = rho0 * w0;
                q[4][idx] = p0 / (gamma - 1.0) + 0.5 * rho0 * (u0 * u0 + v0 * v0 + w0 * w0);
            }
}

/* ---------------------------------------------------------- statistics --- */
/* postproc::solveQ (postproc.cpp:736-930).  Gradients are the primitives'
 * derivatives by each direction's differential scheme (solveGrad -> the
 * operator's differential scheme, periodic halos; postproc.cpp:2285-2297); the per-cell expressions and the (k, j, i) summation order follow
 * postproc.cpp:805-853, the field averages MPICommunicator.cpp:161-185. */
void or_stats(const or_box *b, const double *const q[5], double out[OR_NSTATS]) {
    const long N = (long)b->nx * b->ny * b->nz;
    double *prim[8], *g[9], *qf[16];
    double *blk_prim = alloc_fields(8, N, prim);
    double *blk_g = alloc_fields(9, N, g);
    double *blk_q = alloc_fields(16, N, qf);
    or_con2prim(b, q, prim);
    const double *src[3] = {prim[1], prim[2], prim[3]};
    for (int v = 0; v < 3; ++v)
        for (int d = 0; d < 3; ++d) cd_direction(b, d, src[v], g[v * 3 + d]);
    const double non_dim_T_ref = b->t_ref / b->t_inf;
    double u_rms_aver = 0.0, miu_aver = 0.0, rho_bar = 0.0, div_aver = 0.0, alpha_aver = 0.0;
    double Skew2 = 0.0, Skew3 = 0.0, diss = 0.0;
    for (int k = 0; k < b->nz; ++k)
        for (int j = 0; j < b->ny; ++j)
            for (int i = 0; i < b->nx; ++i) {
                long n = i + (long)b->nx * (j + (long)b->ny * k);
                double u0 = prim[1][n], u1 = prim[2][n], u2 = prim[3][n];
                double ux = g[0][n], uy = g[1][n], uz = g[2][n];
                double vx = g[3][n], vy = g[4][n], vz = g[5][n];
                double wx = g[6][n], wy = g[7][n], wz = g[8][n];
                double w0 = wy - vz, w1 = uz - wx, w2 = vx - uy;
                double q0 = ux * vy + ux * wz + vy * wz - uy * vx - uz * wx - vz * wy;
                for (int c = 0; c < 9; ++c) qf[c][n] = g[c][n];
                qf[9][n] = w0;
                qf[10][n] = w1;
                qf[11][n] = w2;
                qf[12][n] = (w0 * w0 + w1 * w1 + w2 * w2) * 0.5;
                qf[13][n] = q0;
                qf[14][n] = w0 * u0 + w1 * u1 + w2 * u2;
                qf[15][n] = 0.5 * prim[0][n] * (u0 * u0 + u1 * u1 + u2 * u2);
                u_rms_aver += (u0 * u0 + u1 * u1 + u2 * u2) / 3.0;
                div_aver += (ux * ux + vy * vy + wz * wz) / 3.0;
                Skew3 += (pow(ux, 3.0) + pow(vy, 3.0) + pow(wz, 3.0)) / 3.0;
                Skew2 += (ux * ux + vy * vy + wz * wz) / 3.0;
                alpha_aver += prim[7][n];
                double T = prim[5][n];
                miu_aver += (1.0 + non_dim_T_ref) / (T + non_dim_T_ref) * pow(T, 1.5);
                rho_bar += prim[0][n];
                double miu, coeff, th = ux + vy + wz;
                viscosity(b, T, &miu, &coeff);
                diss += miu * (w0 * w0 + w1 * w1 + w2 * w2 + 4.0 / 3.0 * th * th);
            }
    for (int c = 0; c < 16; ++c) {
        double sum = 0.0;
        for (long n = 0; n < N; ++n) sum += qf[c][n];
        out[c] = sum / (double)(int)N;
    }
    const double NN = (double)(int)N;
    u_rms_aver /= NN;
    div_aver /= NN;
    miu_aver /= NN;
    rho_bar /= NN;
    Skew3 /= NN;
    Skew2 /= NN;
    alpha_aver /= NN;
    double skew = Skew3 / pow(Skew2, 1.5);
    double lambda = sqrt(u_rms_aver / div_aver);
    double Re_lambda = sqrt(u_rms_aver) * lambda * rho_bar / miu_aver * b->reynolds;
    double tau_t = lambda / sqrt(u_rms_aver);
    out[16] = sqrt(u_rms_aver);
    out[17] = sqrt(u_rms_aver * 3.0) / alpha_aver;
    out[18] = sqrt(div_aver);
    out[19] = miu_aver;
    out[20] = Re_lambda;
    out[21] = lambda;
    out[22] = rho_bar;
    out[23] = tau_t;
    out[24] = skew;
    out[25] = diss / NN;
    free(blk_prim);
    free(blk_g);
    free(blk_q);
}
