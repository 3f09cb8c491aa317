// Device-side building blocks of the NUC3d RHS: WENO5 reconstructions, CD6,
// viscosity models and the box description passed to every kernel.
//
// Template parameter B is the "bulk" arithmetic type (double for the FP64
// path, float for the mixed path).  The conserved state is always double.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace nuc3d {

enum : unsigned {
    QK_ZETA_EIGEN = 0x1u,
    QK_WENOZ_BETA2 = 0x2u,
    QK_OFFDIAG_DIV = 0x4u,
    QK_FABS_PRESSURE = 0x8u,
    QK_CRWENO_BOUNDED = 0x10u,
};

enum : int {
    SCHEME_JS = 0,
    SCHEME_Z = 1,
    SCHEME_CR = 2,
    SCHEME_W7 = 3,
    SCHEME_HC = 4,
    SCHEME_H77 = 5,
    SCHEME_H78 = 6,
    SCHEME_W3 = 7,
    SCHEME_U1 = 8
};

// reconstruction stencil half-width (the reference's bufferSize,
// fieldOperator.cpp:128-175): 4 cells for weno7js and the hccs family, 3 for
// the WENO5 family, 2 for weno3js, 1 for upwind1st
__host__ __device__ constexpr int scheme_halo(int scheme) {
    return scheme == SCHEME_W3 ? 2 : (scheme == SCHEME_U1 ? 1 : (scheme >= SCHEME_W7 ? 4 : 3));
}
enum : int { VISC_SUTHERLAND = 0, VISC_CONSTANT = 1, VISC_POWERLAW = 2 };
// differential schemes of the viscous terms (Method.in scheme_*_vis,
// fieldOperator.cpp:301-375): centraldifference6th / 2nd / 8th
enum : int { VIS_CD6 = 0, VIS_CD2 = 1, VIS_CD8 = 2 };
enum : int { RIEMANN_LF = 0, RIEMANN_AUSM = 1, RIEMANN_AUSMP = 2 };

// Everything a kernel needs to know about one periodic box.
struct BoxParams {
    int n[3];            // nx, ny, nz
    long long N;         // nx*ny*nz
    long long stride[3]; // 1, nx, nx*ny
    double d[3];         // dx, dy, dz
    double inv_d[3];     // 1/dx, 1/dy, 1/dz
    double gamma, mach, reynolds, prandtl, tref_nd, powerlaw_exp;
    double cfl;
    int visc_model, navier_stokes;
    unsigned quirks;
    int scheme[3];
    int riemann;  // RIEMANN_LF / _AUSM / _AUSMP
    int vis[3];   // VIS_CD6 / _CD2 / _CD8 per direction
    // each direction's differential scheme as the coefficients of
    // f(i+m) - f(i-m), m = 1..4 (zero beyond the scheme's reach)
    double vcoef[3][4];
};

// Field pointers of one box.  q: conserved state (double); w: primitives in
// the bulk type (u, v, w, p, c, T); r: inviscid RHS accumulator (bulk);
// vf: viscous flux components (bulk) tau_xx, tau_xy, tau_xz, tau_yy, tau_yz,
// tau_zz, E_x, E_y, E_z.
template <typename B>
struct Fields {
    const double *q[5];
    B *w[6];
    B *r[5];
    B *vf[9];
};

// schemes.hpp:14-36 constants
struct K {
    static constexpr double A00 = 1.0 / 3.0, A01 = -7.0 / 6.0, A02 = 11.0 / 6.0;
    static constexpr double A10 = -1.0 / 6.0, A11 = 5.0 / 6.0, A12 = 1.0 / 3.0;
    static constexpr double A20 = 1.0 / 3.0, A21 = 5.0 / 6.0, A22 = -1.0 / 6.0;
    static constexpr double C0 = 0.1, C1 = 0.6, C2 = 0.3;      // WENO5 linear weights
    static constexpr double CR0 = 0.2, CR1 = 0.5, CR2 = 0.3;   // CRWENO5 linear weights
    static constexpr double G0 = 13.0 / 12.0, G1 = 1.0 / 4.0;
    static constexpr double SG0 = 1.0408329997330663;  // sqrt(13/12)
    static constexpr double CD1 = 3.0 / 4.0, CD2 = -3.0 / 20.0, CD3 = 1.0 / 60.0;
    // schemes.hpp:36, :42
    static constexpr double C81 = 4.0 / 5.0, C82 = -1.0 / 5.0, C83 = 4.0 / 105.0,
                            C84 = -1.0 / 280.0;
    static constexpr double C21 = 0.5;
};

__device__ __forceinline__ int wrap(int c, int n) {
    // periodic index for c in [-n, 2n)
    return c < 0 ? c + n : (c >= n ? c - n : c);
}

// Smoothness indicators of the three 3-cell sub-stencils (schemes.hpp
// gamma0/gamma1 form, weno5js.cpp:75-82).  f0 is the farthest-upwind cell.
template <typename B>
__device__ __forceinline__ void weno5_beta(B f0, B f1, B f2, B f3, B f4, B &is0, B &is1, B &is2,
                                           bool beta2_quirk) {
    const B g0 = B(K::G0), g1 = B(K::G1);
    B d0 = f0 - B(2) * f1 + f2, e0 = f0 - B(4) * f1 + B(3) * f2;
    B d1 = f1 - B(2) * f2 + f3, e1 = f1 - f3;
    // weno5z.cpp:80 reads f[i]-2f[i+1]+f[i+1] on inner '+' faces
    B d2 = beta2_quirk ? (f2 - B(2) * f3 + f3) : (f2 - B(2) * f3 + f4);
    B e2 = B(3) * f2 - B(4) * f3 + f4;
    is0 = g0 * d0 * d0 + g1 * e0 * e0;
    is1 = g0 * d1 * d1 + g1 * e1 * e1;
    is2 = g0 * d2 * d2 + g1 * e2 * e2;
}

template <typename B>
__device__ __forceinline__ void weno5_candidates(B f0, B f1, B f2, B f3, B f4, B &q0, B &q1,
                                                 B &q2) {
    q0 = B(K::A00) * f0 + B(K::A01) * f1 + B(K::A02) * f2;
    q1 = B(K::A10) * f1 + B(K::A11) * f2 + B(K::A12) * f3;
    q2 = B(K::A20) * f2 + B(K::A21) * f3 + B(K::A22) * f4;
}

// Explicitly rounded arithmetic.  The sweep kernels come in variants that
// unroll different numbers of faces per thread; with free FMA contraction the
// compiler shares products across unrolled faces differently per variant and
// the results would differ in the last bits.  Spelling every operation with a
// rounding intrinsic fixes the operation sequence, so all variants (and hence
// a box alone or in any batch) give bitwise identical results.
__device__ __forceinline__ double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double div_(double a, double b) { return __ddiv_rn(a, b); }

// ---- packed FP32 pairs (sm_100 f32x2 arithmetic) ----
// Component-wise each is the correctly rounded scalar operation of the same
// name (fma_, mul_, add_, sub_), so a pair of reconstructions computed
// together gives bitwise the values of the two computed apart, in half the
// FP32 instructions.  a - b is formed as fma(b, -1, a): one rounding, as the
// subtraction.
__device__ __forceinline__ float2 splat2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 fma2_(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2_(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2_(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2_(float2 a, float2 b) {
    return __ffma2_rn(b, splat2(-1.0f), a);
}
__device__ __forceinline__ float2 dd2_of(float2 D) {
    const float2 t = mul2_(splat2(float(2.0 * K::SG0)), D);
    return mul2_(t, t);
}

// second difference f0 - 2 f1 + f2
template <typename B>
__device__ __forceinline__ B d2_(B f0, B f1, B f2) {
    return add_(fma_(B(-2), f1, f0), f2);
}

// sqrt(13/12) (f0 - 2 f1 + f2): with it and half the first-difference term
// e, a smoothness indicator (schemes.hpp:33-34) is the two-operation
// d^2 + e^2 (one multiply, one FMA)
template <typename B>
__device__ __forceinline__ B sd2_(B f0, B f1, B f2) {
    const B c = B(K::SG0), m2c = B(-2.0 * K::SG0);
    return fma_(c, f0, fma_(m2c, f1, mul_(c, f2)));
}

// FP64 reciprocal of a nonzero normal x (weight denominators, line-solve
// pivots, 1/rho): the hardware's approximate reciprocal (PTX
// rcp.approx.ftz.f64, about 2^-20 relative error) refined by two
// Newton-Raphson steps r <- r + r (1 - x r), each squaring the relative
// error, so the result is within an ulp of 1/x (not always the correctly
// rounded value; an ulp is far below the 1e-12 parity bar).  Measured at
// 256^3: WENO5-Z / WENO5-JS FP64 sweeps 4-6 % faster than with the correctly
// rounded reciprocal.  (The WENO7 faces keep __drcp_rn: with this one their
// uncapped y/z kernels took 158 instead of 128 registers and ran 7 % slower.)
__device__ __forceinline__ double drcp_nr(double x) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    r = fma_(r, fma_(-x, r, 1.0), r);
    return fma_(r, fma_(-x, r, 1.0), r);
}

// Fast FP32 reciprocal (one MUFU op, ~1 ulp): the weights only need FP32
// accuracy in the mixed path.
__device__ __forceinline__ float frcp_fast(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// WENO5-JS nonlinear combination (weno5js.cpp:97-108), eps = 1e-6, p = 2:
// alpha_k = c_k/(eps+beta_k)^2 normalised by their sum.  FP64 writes it with a
// single reciprocal by multiplying through with s0^2 s1^2 s2^2 (an exact
// rearrangement); FP32 uses fast reciprocals.
__device__ __forceinline__ double weno_js_combine(double is0, double is1, double is2, double q0,
                                                  double q1, double q2) {
    const double ss = 1.0e-6;
    double s0 = add_(ss, is0), s1 = add_(ss, is1), s2 = add_(ss, is2);
    s0 = mul_(s0, s0);
    s1 = mul_(s1, s1);
    s2 = mul_(s2, s2);
    double w0 = mul_(K::C0, mul_(s1, s2)), w1 = mul_(K::C1, mul_(s0, s2));
    double w2 = mul_(K::C2, mul_(s0, s1));
    return mul_(fma_(w2, q2, fma_(w1, q1, mul_(w0, q0))), drcp_nr(add_(add_(w0, w1), w2)));
}
__device__ __forceinline__ float weno_js_combine(float is0, float is1, float is2, float q0,
                                                 float q1, float q2) {
    const float ss = 1.0e-6f;
    float r0 = frcp_fast(add_(ss, is0)), r1 = frcp_fast(add_(ss, is1)), r2 = frcp_fast(add_(ss, is2));
    float a0 = mul_(mul_(float(K::C0), r0), r0), a1 = mul_(mul_(float(K::C1), r1), r1);
    float a2 = mul_(mul_(float(K::C2), r2), r2);
    return mul_(fma_(a2, q2, fma_(a1, q1, mul_(a0, q0))), frcp_fast(add_(add_(a0, a1), a2)));
}

// WENO5-Z combination (weno5z.cpp:96-109), eps = 1e-40, p = 2:
// alpha_k = c_k (1 + (tau/(beta_k+eps))^2), tau = |beta2 - beta0|.
__device__ __forceinline__ double weno_z_combine(double is0, double is1, double is2, double q0,
                                                 double q1, double q2) {
    const double ss = 1.0e-40;
    double tau = fabs(sub_(is2, is0));
    double t2 = mul_(tau, tau);
    double s0 = add_(is0, ss), s1 = add_(is1, ss), s2 = add_(is2, ss);
    s0 = mul_(s0, s0);
    s1 = mul_(s1, s1);
    s2 = mul_(s2, s2);
    // alpha_k * s0^2 s1^2 s2^2 = c_k (s_k^2 + tau^2) prod_{j!=k} s_j^2
    double w0 = mul_(mul_(K::C0, add_(s0, t2)), mul_(s1, s2));
    double w1 = mul_(mul_(K::C1, add_(s1, t2)), mul_(s0, s2));
    double w2 = mul_(mul_(K::C2, add_(s2, t2)), mul_(s0, s1));
    return mul_(fma_(w2, q2, fma_(w1, q1, mul_(w0, q0))), drcp_nr(add_(add_(w0, w1), w2)));
}
__device__ __forceinline__ float weno_z_combine(float is0, float is1, float is2, float q0, float q1,
                                                float q2) {
    // 1e-40 is below FP32's normal range; 1e-30 keeps the ratio finite and
    // only differs where a sub-stencil is exactly constant.  The ratio is
    // capped at 1e15 so that alpha (<= 1e30) times a candidate stays far
    // below FP32's 3.4e38 (a capped weight carries the face anyway).
    const float ss = 1.0e-30f, cap = 1.0e15f;
    float tau = fabsf(sub_(is2, is0));
    float t0 = fminf(mul_(tau, frcp_fast(add_(is0, ss))), cap);
    float t1 = fminf(mul_(tau, frcp_fast(add_(is1, ss))), cap);
    float t2 = fminf(mul_(tau, frcp_fast(add_(is2, ss))), cap);
    float a0 = mul_(float(K::C0), fma_(t0, t0, 1.0f));
    float a1 = mul_(float(K::C1), fma_(t1, t1, 1.0f));
    float a2 = mul_(float(K::C2), fma_(t2, t2, 1.0f));
    return mul_(fma_(a2, q2, fma_(a1, q1, mul_(a0, q0))), frcp_fast(add_(add_(a0, a1), a2)));
}

// The same combinations in offset form for the sweeps: with dq_k = q_k - f2
// the face is f2 + sum(w_k dq_k) / sum(w_k), which saves the candidates'
// common part and keeps the rounding relative to the local variation.  The
// linear weights are 0.1 (1, 6, 3); the 0.1 cancels in the ratio and the 6
// and 3 go with the candidates, so the caller passes g = (dq0, 6 dq1, 3 dq2)
// and the face is f2 + (w0 g0 + w1 g1 + w2 g2) / (w0 + 6 w1 + 3 w2) with w_k
// the weights without their linear factor.  The indicators arrive scaled by
// 4 (is_k = 4 beta_k, see weno5_face_dq) and eps with them, an exact scaling
// that leaves every weight ratio bitwise unchanged.  WENO5-Z's
// (beta + 1e-40)^2 is formed as beta^2 + 1e-80 (the cross term is below
// 1e-40 of beta).
__device__ __forceinline__ double weno_js_combine_dq(double is0, double is1, double is2,
                                                     double g0, double g1, double g2,
                                                     double f2) {
    const double ss = 4.0 * 1.0e-6;  // 4 eps
    double s0 = add_(ss, is0), s1 = add_(ss, is1), s2 = add_(ss, is2);
    s0 = mul_(s0, s0);
    s1 = mul_(s1, s1);
    s2 = mul_(s2, s2);
    const double w0 = mul_(s1, s2), w1 = mul_(s0, s2), w2 = mul_(s0, s1);
    return fma_(fma_(w2, g2, fma_(w1, g1, mul_(w0, g0))),
                drcp_nr(fma_(6.0, w1, fma_(3.0, w2, w0))), f2);
}
__device__ __forceinline__ float weno_js_combine_dq(float is0, float is1, float is2, float g0,
                                                    float g1, float g2, float f2) {
    const float ss = 4.0f * 1.0e-6f;  // 4 eps
    float r0 = frcp_fast(add_(ss, is0)), r1 = frcp_fast(add_(ss, is1)), r2 = frcp_fast(add_(ss, is2));
    const float a0 = mul_(r0, r0), a1 = mul_(r1, r1), a2 = mul_(r2, r2);
    return fma_(fma_(a2, g2, fma_(a1, g1, mul_(a0, g0))),
                frcp_fast(fma_(6.0f, a1, fma_(3.0f, a2, a0))), f2);
}
__device__ __forceinline__ double weno_z_combine_dq(double is0, double is1, double is2,
                                                    double g0, double g1, double g2,
                                                    double f2) {
    const double ss2 = 16.0 * 1.0e-80;  // (4 eps)^2, eps = 1e-40
    const double tau = sub_(is2, is0);
    const double t2 = mul_(tau, tau);
    double s0 = fma_(is0, is0, ss2), s1 = fma_(is1, is1, ss2), s2 = fma_(is2, is2, ss2);
    // alpha_k / c_k * s0^2 s1^2 s2^2 = (s_k^2 + tau^2) prod_{j!=k} s_j^2
    //                                = P + tau^2 prod_{j!=k} s_j^2,  P = s0^2 s1^2 s2^2
    // (three products, one more for P, three FMAs)
    const double p12 = mul_(s1, s2), p02 = mul_(s0, s2), p01 = mul_(s0, s1);
    const double P = mul_(s0, p12);
    const double w0 = fma_(t2, p12, P), w1 = fma_(t2, p02, P), w2 = fma_(t2, p01, P);
    return fma_(fma_(w2, g2, fma_(w1, g1, mul_(w0, g0))),
                drcp_nr(fma_(6.0, w1, fma_(3.0, w2, w0))), f2);
}
__device__ __forceinline__ float weno_z_combine_dq(float is0, float is1, float is2, float g0,
                                                   float g1, float g2, float f2) {
    const float ss = 4.0f * 1.0e-30f, cap = 1.0e15f;  // 4 eps
    float tau = fabsf(sub_(is2, is0));
    float t0 = fminf(mul_(tau, frcp_fast(add_(is0, ss))), cap);
    float t1 = fminf(mul_(tau, frcp_fast(add_(is1, ss))), cap);
    float t2 = fminf(mul_(tau, frcp_fast(add_(is2, ss))), cap);
    const float a0 = fma_(t0, t0, 1.0f), a1 = fma_(t1, t1, 1.0f), a2 = fma_(t2, t2, 1.0f);
    return fma_(fma_(a2, g2, fma_(a1, g1, mul_(a0, g0))),
                frcp_fast(fma_(6.0f, a1, fma_(3.0f, a2, a0))), f2);
}

// One WENO5 face (either scheme) from the sliding window's differences:
// a_ij = f_i - f_j of the upwind-oriented stencil f0..f4, the second
// differences D0 = f0 - 2 f1 + f2 and D2 = f2 - 2 f3 + f4, and dd_k (the
// indicators' first terms, carried from face to face).  The indicators are formed times 4 (schemes.hpp:33-34 with the 1/4 of the
// second term absorbed): with E_k the second terms' differences,
//   E0 = D0 + 2 a21,  E1 = -(a21 + a32) (its sign drops in the square),
//   E2 = D2 - 2 a32,   4 beta_k = dd_k + E_k^2,  dd_k = 4 (13/12) D_k^2,
// and the candidates (schemes.hpp:14-18) as f2 + dq_k:
//   dq0 = D0/3 + a21/2,  6 dq1 = a21 + 2 a32,  3 dq2 = 2 a32 - a43/2.
template <int SCHEME, typename B>
__device__ __forceinline__ B weno5_face_dq(B f2, B a21, B a32, B a43, B D0, B D2, B dd0, B dd1,
                                           B dd2) {
    const B h = B(0.5);
    const B e0 = fma_(B(2), a21, D0);
    const B e1 = add_(a21, a32);
    const B e2 = fma_(B(-2), a32, D2);
    const B is0 = fma_(e0, e0, dd0), is1 = fma_(e1, e1, dd1), is2 = fma_(e2, e2, dd2);
    const B g0 = fma_(B(1.0 / 3.0), D0, mul_(h, a21));
    const B g1 = fma_(B(2), a32, a21);
    const B g2 = fma_(B(2), a32, mul_(B(-0.5), a43));
    if (SCHEME == SCHEME_Z) return weno_z_combine_dq(is0, is1, is2, g0, g1, g2, f2);
    return weno_js_combine_dq(is0, is1, is2, g0, g1, g2, f2);
}

// Two FP32 faces at once (component x: one stencil, y: another), packed:
// component-wise the operations of weno5_face_dq<SCHEME, float> with
// weno_z_combine_dq / weno_js_combine_dq, in the same order, so each
// component is bitwise that face.  The reciprocals, |.| and min stay scalar.
template <int SCHEME>
__device__ __forceinline__ float2 weno5_face_dq2(float2 f2, float2 a21, float2 a32, float2 a43,
                                                 float2 D0, float2 D2, float2 dd0, float2 dd1,
                                                 float2 dd2) {
    const float2 e0 = fma2_(splat2(2.0f), a21, D0);
    const float2 e1 = add2_(a21, a32);
    const float2 e2 = fma2_(splat2(-2.0f), a32, D2);
    const float2 is0 = fma2_(e0, e0, dd0), is1 = fma2_(e1, e1, dd1), is2 = fma2_(e2, e2, dd2);
    const float2 g0 = fma2_(splat2(float(1.0 / 3.0)), D0, mul2_(splat2(0.5f), a21));
    const float2 g1 = fma2_(splat2(2.0f), a32, a21);
    const float2 g2 = fma2_(splat2(2.0f), a32, mul2_(splat2(-0.5f), a43));
    float2 a0, a1, a2;
    if (SCHEME == SCHEME_Z) {
        const float ss = 4.0f * 1.0e-30f, cap = 1.0e15f;
        const float2 d = sub2_(is2, is0);
        const float2 tau = make_float2(fabsf(d.x), fabsf(d.y));
        const float2 q0 = add2_(is0, splat2(ss)), q1 = add2_(is1, splat2(ss)),
                     q2 = add2_(is2, splat2(ss));
        float2 t0 = mul2_(tau, make_float2(frcp_fast(q0.x), frcp_fast(q0.y)));
        float2 t1 = mul2_(tau, make_float2(frcp_fast(q1.x), frcp_fast(q1.y)));
        float2 t2 = mul2_(tau, make_float2(frcp_fast(q2.x), frcp_fast(q2.y)));
        t0 = make_float2(fminf(t0.x, cap), fminf(t0.y, cap));
        t1 = make_float2(fminf(t1.x, cap), fminf(t1.y, cap));
        t2 = make_float2(fminf(t2.x, cap), fminf(t2.y, cap));
        a0 = fma2_(t0, t0, splat2(1.0f));
        a1 = fma2_(t1, t1, splat2(1.0f));
        a2 = fma2_(t2, t2, splat2(1.0f));
    } else {
        const float ss = 4.0f * 1.0e-6f;
        const float2 q0 = add2_(splat2(ss), is0), q1 = add2_(splat2(ss), is1),
                     q2 = add2_(splat2(ss), is2);
        const float2 r0 = make_float2(frcp_fast(q0.x), frcp_fast(q0.y));
        const float2 r1 = make_float2(frcp_fast(q1.x), frcp_fast(q1.y));
        const float2 r2 = make_float2(frcp_fast(q2.x), frcp_fast(q2.y));
        a0 = mul2_(r0, r0);
        a1 = mul2_(r1, r1);
        a2 = mul2_(r2, r2);
    }
    const float2 num = fma2_(a2, g2, fma2_(a1, g1, mul2_(a0, g0)));
    const float2 den = fma2_(splat2(6.0f), a1, fma2_(splat2(3.0f), a2, a0));
    return fma2_(num, make_float2(frcp_fast(den.x), frcp_fast(den.y)), f2);
}

// 4 (13/12) D^2 as (2 sqrt(13/12) D)^2 (the sweeps' indicators are formed
// times 4)
template <typename B>
__device__ __forceinline__ B dd_of(B D) {
    const B t = mul_(B(2.0 * K::SG0), D);
    return mul_(t, t);
}

// WENO5 smoothness indicators times 4 of the upwind-oriented stencil
// f0..f4 (schemes.hpp:33-34), from first and second differences:
// 4 beta_k = 4 (13/12) D_k^2 + E_k^2 with D_k the sub-stencil's second
// difference and E0 = D0 + 2 (f2 - f1), E1 = (f2 - f1) + (f3 - f2),
// E2 = D2 - 2 (f3 - f2).
template <typename B>
__device__ __forceinline__ void weno5_beta4(B f0, B f1, B f2, B f3, B f4, B &is0, B &is1, B &is2) {
    const B a10 = sub_(f1, f0), a21 = sub_(f2, f1), a32 = sub_(f3, f2), a43 = sub_(f4, f3);
    const B D0 = sub_(a21, a10), D1 = sub_(a32, a21), D2 = sub_(a43, a32);
    const B e0 = fma_(B(2), a21, D0), e1 = add_(a21, a32), e2 = fma_(B(-2), a32, D2);
    is0 = fma_(e0, e0, dd_of(D0));
    is1 = fma_(e1, e1, dd_of(D1));
    is2 = fma_(e2, e2, dd_of(D2));
}

template <int SCHEME, typename B>
__device__ __forceinline__ B weno_combine(B is0, B is1, B is2, B q0, B q1, B q2) {
    if (SCHEME == SCHEME_Z) return weno_z_combine(is0, is1, is2, q0, q1, q2);
    return weno_js_combine(is0, is1, is2, q0, q1, q2);
}

// Face values from an upwind-oriented 5-cell stencil (f0 farthest upwind).
template <typename B>
__device__ __forceinline__ B weno5js_face(B f0, B f1, B f2, B f3, B f4) {
    B is0, is1, is2, q0, q1, q2;
    weno5_beta(f0, f1, f2, f3, f4, is0, is1, is2, false);
    weno5_candidates(f0, f1, f2, f3, f4, q0, q1, q2);
    return weno_js_combine(is0, is1, is2, q0, q1, q2);
}
template <typename B>
__device__ __forceinline__ B weno5z_face(B f0, B f1, B f2, B f3, B f4, bool beta2_quirk) {
    B is0, is1, is2, q0, q1, q2;
    weno5_beta(f0, f1, f2, f3, f4, is0, is1, is2, beta2_quirk);
    weno5_candidates(f0, f1, f2, f3, f4, q0, q1, q2);
    return weno_z_combine(is0, is1, is2, q0, q1, q2);
}

template <int SCHEME, typename B>
__device__ __forceinline__ B weno5_face(B f0, B f1, B f2, B f3, B f4, bool beta2_quirk) {
    if (SCHEME == SCHEME_Z) return weno5z_face(f0, f1, f2, f3, f4, beta2_quirk);
    return weno5js_face(f0, f1, f2, f3, f4);
}

// --------------------------------------------------------- flux splitting --
// Point-wise split of the DIR flux of one cell into F+ (reconstructed
// upwind '+') and F- ('-').  FP64, each operation explicitly rounded in the
// reference's order.
//   LF    (physicsModel.cpp:546-565): F+- = (F(Q) +- lambda Q) / 2,
//         lambda = |u_n| + c.
//   AUSM  (:777-929), AUSMp (:1027-1178), with m = u_n / c:
//         F+- = (M+-(m) c) Q + p+-(m) e_n + (M+-(m) c) p e_E, the Mach
//         polynomials M+- and pressure weights p+- of :1181-1278.
struct SplitCell {
    double a[2];  // LF: u_n and lambda; AUSM: M+ c and M- c
    double p;     // pressure
    double pn[2]; // AUSM: p+ and p- (the normal-momentum terms)
};

__device__ __forceinline__ double sq_(double x) { return mul_(x, x); }

__device__ __forceinline__ void split_prepare(int riemann, double un, double p, double c,
                                              SplitCell &s) {
    s.p = p;
    if (riemann == RIEMANN_LF) {
        s.a[0] = un;
        s.a[1] = add_(fabs(un), c);
        return;
    }
    // m = u_n / c by a correctly rounded reciprocal (within an ulp of the
    // reference's division); no division is inlined into the sweeps.  For
    // |m| >= 1 the pressure weights 0.5 p (m +- |m|) / m are p or 0 exactly
    // in real arithmetic (the reference's rounding of them is within an ulp).
    const double m = mul_(un, __drcp_rn(c));
    const double am = fabs(m);
    double mp, mm, pp, pm;
    if (am < 1.0) {
        const double q2 = sq_(sub_(mul_(m, m), 1.0));
        mp = add_(mul_(0.25, sq_(add_(m, 1.0))), mul_(0.125, q2));
        mm = sub_(mul_(-0.25, sq_(sub_(m, 1.0))), mul_(0.125, q2));
        if (riemann == RIEMANN_AUSM) {
            pp = mul_(mul_(p, add_(m, 1.0)), 0.5);
            pm = mul_(mul_(-p, sub_(m, 1.0)), 0.5);
        } else {
            const double t = mul_(mul_(0.1875, m), q2);
            pp = mul_(p, add_(mul_(mul_(0.25, sq_(add_(m, 1.0))), sub_(2.0, m)), t));
            pm = mul_(p, sub_(mul_(mul_(0.25, sq_(sub_(m, 1.0))), add_(2.0, m)), t));
        }
    } else {
        mp = mul_(0.5, add_(m, am));
        mm = mul_(0.5, sub_(m, am));
        pp = m > 0.0 ? p : 0.0;
        pm = m > 0.0 ? 0.0 : p;
    }
    s.a[0] = mul_(mp, c);
    s.a[1] = mul_(mm, c);
    s.pn[0] = pp;
    s.pn[1] = pm;
}

// F+ and F- of equation e (0..4) of a cell with conserved value qe
template <int DIR>
__device__ __forceinline__ void split_eq(int riemann, const SplitCell &s, int e, double qe,
                                         double &fp, double &fm) {
    if (riemann == RIEMANN_LF) {
        // F+- = F/2 +- (lambda/2) q, the halves taken first (exact)
        const double hun = mul_(0.5, s.a[0]), hlam = mul_(0.5, s.a[1]);
        double hf;
        if (e == 4)
            hf = mul_(hun, add_(qe, s.p));
        else if (e == 1 + DIR)
            hf = fma_(hun, qe, mul_(0.5, s.p));
        else
            hf = mul_(hun, qe);
        fp = fma_(hlam, qe, hf);
        fm = fma_(-hlam, qe, hf);
        return;
    }
    fp = mul_(s.a[0], qe);
    fm = mul_(s.a[1], qe);
    if (e == 1 + DIR) {
        fp = add_(fp, s.pn[0]);
        fm = add_(fm, s.pn[1]);
    } else if (e == 4) {
        fp = add_(fp, mul_(s.a[0], s.p));
        fm = add_(fm, mul_(s.a[1], s.p));
    }
}

// ------------------------------------------------------------------ WENO7 --
// The reference's weno7js face (weno7js.cpp:79-126 for '+', :179-226 for
// '-'; the boundary forms :227-824 are the same expression on halo cells).
// f[0..6] is the upwind-oriented 7-cell stencil (f[0] farthest upwind).
// Smoothness indicators: Balsara-Shu integer quadratic forms of the four
// 4-cell sub-stencils (weno7js.cpp:83-106); candidates: the four cubic
// interpolants (coeff_weno7_alpha, schemes.hpp); weights of Z type,
// alpha_k = c_k (1 + (tau7/(eps + beta_k))^2) with tau7 = |beta0 - beta3|,
// eps = 1e-20 and c = {1, 12, 18, 4}/35 (weno7js.cpp:107-123).
struct K7 {
    static constexpr double C0 = 1.0 / 35.0, C1 = 12.0 / 35.0, C2 = 18.0 / 35.0, C3 = 4.0 / 35.0;
};

// beta of a 4-cell sub-stencil a, b, c, d in the reference's nested form
// a(k00 a + k01 b + k02 c + k03 d) + b(k11 b + k12 c + k13 d) + c(k22 c + k23 d)
// + k33 d^2.  The form cancels heavily (its coefficients sum to zero, so
// terms of size 1e4 f^2 cancel down to 1e2 (f' dx)^2): the rounding of each
// operation shows in beta.  FP64 therefore evaluates it unfused, in the
// reference's left-to-right order, which keeps the faces within ~1e-14 of
// the reference where a fused evaluation drifts to ~1e-12 in the RHS.
__device__ __forceinline__ double weno7_form(double a, double b, double c, double d, double k00,
                                             double k01, double k02, double k03, double k11,
                                             double k12, double k13, double k22, double k23,
                                             double k33) {
    double ta = add_(add_(add_(mul_(k00, a), mul_(k01, b)), mul_(k02, c)), mul_(k03, d));
    double tb = add_(add_(mul_(k11, b), mul_(k12, c)), mul_(k13, d));
    double tc = add_(mul_(k22, c), mul_(k23, d));
    return add_(add_(add_(mul_(a, ta), mul_(b, tb)), mul_(c, tc)), mul_(mul_(k33, d), d));
}
__device__ __forceinline__ void weno7_parts(double f0, double f1, double f2, double f3, double f4,
                                            double f5, double f6, double is[4], double q[4]) {
    using B = double;
    is[0] = weno7_form(f0, f1, f2, f3, 547.0, -3882.0, 4642.0, -1854.0, 7043.0, -17246.0,
                       7042.0, 11003.0, -9402.0, 2107.0);
    is[1] = weno7_form(f1, f2, f3, f4, 267.0, -1642.0, 1602.0, -494.0, 2843.0, -5966.0, 1922.0,
                       3443.0, -2522.0, 547.0);
    is[2] = weno7_form(f2, f3, f4, f5, 547.0, -2522.0, 1922.0, -494.0, 3443.0, -5966.0, 1602.0,
                       2843.0, -1642.0, 267.0);
    is[3] = weno7_form(f3, f4, f5, f6, 2107.0, -9402.0, 7042.0, -1854.0, 11003.0, -17246.0,
                       4642.0, 7043.0, -3882.0, 547.0);
    // cubic candidates (1/12)(...): rows of coeff_weno7_alpha
    q[0] = fma_(B(-3.0 / 12.0), f0, fma_(B(13.0 / 12.0), f1, fma_(B(-23.0 / 12.0), f2,
                                                                   mul_(B(25.0 / 12.0), f3))));
    q[1] = fma_(B(1.0 / 12.0), f1, fma_(B(-5.0 / 12.0), f2, fma_(B(13.0 / 12.0), f3,
                                                                  mul_(B(3.0 / 12.0), f4))));
    q[2] = fma_(B(-1.0 / 12.0), f2, fma_(B(7.0 / 12.0), f3, fma_(B(7.0 / 12.0), f4,
                                                                  mul_(B(-1.0 / 12.0), f5))));
    q[3] = fma_(B(3.0 / 12.0), f3, fma_(B(13.0 / 12.0), f4, fma_(B(-5.0 / 12.0), f5,
                                                                  mul_(B(1.0 / 12.0), f6))));
}

// FP64 weights multiplied through by s0^2 s1^2 s2^2 s3^2 (s_k = beta_k + eps),
// an exact rearrangement that needs one reciprocal:
// alpha_k * prod s^2 = c_k (s_k^2 + tau^2) prod_{j != k} s_j^2.
__device__ __forceinline__ double weno7_combine(const double is[4], const double q[4]) {
    const double ss = 1.0e-20;
    double tau = fabs(sub_(is[0], is[3]));
    double t2 = mul_(tau, tau);
    double s0 = add_(ss, is[0]), s1 = add_(ss, is[1]), s2 = add_(ss, is[2]), s3 = add_(ss, is[3]);
    s0 = mul_(s0, s0);
    s1 = mul_(s1, s1);
    s2 = mul_(s2, s2);
    s3 = mul_(s3, s3);
    double p01 = mul_(s0, s1), p23 = mul_(s2, s3);
    double w0 = mul_(mul_(K7::C0, add_(s0, t2)), mul_(s1, p23));
    double w1 = mul_(mul_(K7::C1, add_(s1, t2)), mul_(s0, p23));
    double w2 = mul_(mul_(K7::C2, add_(s2, t2)), mul_(s3, p01));
    double w3 = mul_(mul_(K7::C3, add_(s3, t2)), mul_(s2, p01));
    double num = fma_(w3, q[3], fma_(w2, q[2], fma_(w1, q[1], mul_(w0, q[0]))));
    return mul_(num, __drcp_rn(add_(add_(add_(w0, w1), w2), w3)));
}
__device__ __forceinline__ double weno7_face(double f0, double f1, double f2, double f3, double f4,
                                             double f5, double f6) {
    double is[4], q[4];
    weno7_parts(f0, f1, f2, f3, f4, f5, f6, is, q);
    return weno7_combine(is, q);
}

// hccs's WENO7 faces (hccs.cpp:538-980 and its identity rows): the same
// face with hccs's own eps = 1e-40.  FP64 forms the weights through
// reciprocals (alpha_k = c_k (1 + (tau r_k)^2), r_k = 1/(eps + beta_k)): with
// eps = 1e-40 the one-reciprocal product form would multiply four factors
// as small as 1e-80 and underflow.
__device__ __forceinline__ double weno7_face_hc(double f0, double f1, double f2, double f3,
                                                double f4, double f5, double f6) {
    double is[4], q[4];
    weno7_parts(f0, f1, f2, f3, f4, f5, f6, is, q);
    const double ss = 1.0e-40;
    const double tau = fabs(sub_(is[0], is[3]));
    const double c[4] = {K7::C0, K7::C1, K7::C2, K7::C3};
    double a[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double r = mul_(tau, __drcp_rn(add_(ss, is[k])));
        a[k] = mul_(c[k], fma_(r, r, 1.0));
    }
    const double num = fma_(a[3], q[3], fma_(a[2], q[2], fma_(a[1], q[1], mul_(a[0], q[0]))));
    return mul_(num, __drcp_rn(add_(add_(add_(a[0], a[1]), a[2]), a[3])));
}

// FP32 (mixed path): the same indicators and candidates rewritten exactly in
// first and second differences, which removes the cancellation instead of
// ordering it.  With delta_j = f_j - f_{j-1} and sigma_j = delta_j -
// delta_{j-1}, sub-stencil k has u = delta_{k+2}, a = sigma_{k+2},
// b = sigma_{k+3} and
//   beta_k = 240 u^2 + p_k u a + r_k u b + s_k a^2 + t_k a b + v_k b^2
// (the Balsara-Shu forms under that change of variables), and each cubic
// candidate is f3 plus an integer combination of deltas over 12.  Smooth data
// gives beta ~ 240 u^2 with small corrections, so FP32 rounding stays
// relative to the differences, not to the flux itself.
__device__ __forceinline__ float w7_beta(float u, float a, float b, float p, float r, float s,
                                         float t, float v) {
    float tu = fma_(r, b, fma_(p, a, mul_(240.0f, u)));
    float ta = fma_(t, b, mul_(s, a));
    return fma_(u, tu, fma_(a, ta, mul_(mul_(v, b), b)));
}
__device__ __forceinline__ float weno7_face_eps(float f0, float f1, float f2, float f3, float f4,
                                                float f5, float f6, float ss);
__device__ __forceinline__ float weno7_face(float f0, float f1, float f2, float f3, float f4,
                                            float f5, float f6) {
    return weno7_face_eps(f0, f1, f2, f3, f4, f5, f6, 1.0e-20f);
}
// hccs's faces in FP32: 1e-40 is below FP32's normal range, 1e-30 stands in
// (it only matters where a sub-stencil is exactly constant)
__device__ __forceinline__ float weno7_face_hc(float f0, float f1, float f2, float f3, float f4,
                                               float f5, float f6) {
    return weno7_face_eps(f0, f1, f2, f3, f4, f5, f6, 1.0e-30f);
}
__device__ __forceinline__ float weno7_face_eps(float f0, float f1, float f2, float f3, float f4,
                                                float f5, float f6, float ss) {
    float d1 = sub_(f1, f0), d2 = sub_(f2, f1), d3 = sub_(f3, f2);
    float d4 = sub_(f4, f3), d5 = sub_(f5, f4), d6 = sub_(f6, f5);
    float s2 = sub_(d2, d1), s3 = sub_(d3, d2), s4 = sub_(d4, d3), s5 = sub_(d5, d4),
          s6 = sub_(d6, d5);
    float is[4], r[4];
    is[0] = w7_beta(d2, s2, s3, -160.0f, 880.0f, 547.0f, -1854.0f, 2107.0f);
    is[1] = w7_beta(d3, s3, s4, 80.0f, 160.0f, 267.0f, -494.0f, 547.0f);
    is[2] = w7_beta(d4, s4, s5, -160.0f, -80.0f, 547.0f, -494.0f, 267.0f);
    is[3] = w7_beta(d5, s5, s6, -880.0f, 160.0f, 2107.0f, -1854.0f, 547.0f);
    // the forms are positive semi-definite; rounding can leave a flat
    // sub-stencil's value a little below zero, which with eps 1e-30 would turn
    // tau/(eps + beta) into a huge negative number
#pragma unroll
    for (int k = 0; k < 4; ++k) is[k] = fmaxf(is[k], 0.0f);
    // 12 (q_k - f3)
    r[0] = fma_(3.0f, d1, fma_(-10.0f, d2, mul_(13.0f, d3)));
    r[1] = fma_(-1.0f, d2, fma_(4.0f, d3, mul_(3.0f, d4)));
    r[2] = fma_(-1.0f, d5, fma_(6.0f, d4, d3));
    r[3] = fma_(9.0f, d4, fma_(-4.0f, d5, d6));
    const float cap = 1.0e15f;
    const float c[4] = {float(K7::C0), float(K7::C1), float(K7::C2), float(K7::C3)};
    float tau = fabsf(sub_(is[0], is[3]));
    float al[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float t = fminf(mul_(tau, frcp_fast(add_(ss, is[k]))), cap);
        al[k] = mul_(c[k], fma_(t, t, 1.0f));
    }
    float num = fma_(al[3], r[3], fma_(al[2], r[2], fma_(al[1], r[1], mul_(al[0], r[0]))));
    float den = add_(add_(add_(al[0], al[1]), al[2]), al[3]);
    return fma_(mul_(num, frcp_fast(den)), 1.0f / 12.0f, f3);
}

// Two FP32 WENO7 faces at once (component x: one stencil, y: another) on
// the packed f32x2 arithmetic: component-wise the operations of
// weno7_face_eps<float> in the same order, so each component is bitwise that
// face.  The reciprocals, max, |.| and min stay scalar.
__device__ __forceinline__ float2 w7_beta2(float2 u, float2 a, float2 b, float p, float r,
                                           float s, float t, float v) {
    const float2 tu = fma2_(splat2(r), b, fma2_(splat2(p), a, mul2_(splat2(240.0f), u)));
    const float2 ta = fma2_(splat2(t), b, mul2_(splat2(s), a));
    return fma2_(u, tu, fma2_(a, ta, mul2_(mul2_(splat2(v), b), b)));
}
__device__ __forceinline__ float2 weno7_face2(float2 f0, float2 f1, float2 f2, float2 f3,
                                              float2 f4, float2 f5, float2 f6) {
    const float ss = 1.0e-20f;
    const float2 d1 = sub2_(f1, f0), d2 = sub2_(f2, f1), d3 = sub2_(f3, f2);
    const float2 d4 = sub2_(f4, f3), d5 = sub2_(f5, f4), d6 = sub2_(f6, f5);
    const float2 s2 = sub2_(d2, d1), s3 = sub2_(d3, d2), s4 = sub2_(d4, d3), s5 = sub2_(d5, d4),
                 s6 = sub2_(d6, d5);
    float2 is[4], r[4];
    is[0] = w7_beta2(d2, s2, s3, -160.0f, 880.0f, 547.0f, -1854.0f, 2107.0f);
    is[1] = w7_beta2(d3, s3, s4, 80.0f, 160.0f, 267.0f, -494.0f, 547.0f);
    is[2] = w7_beta2(d4, s4, s5, -160.0f, -80.0f, 547.0f, -494.0f, 267.0f);
    is[3] = w7_beta2(d5, s5, s6, -880.0f, 160.0f, 2107.0f, -1854.0f, 547.0f);
#pragma unroll
    for (int k = 0; k < 4; ++k) is[k] = make_float2(fmaxf(is[k].x, 0.0f), fmaxf(is[k].y, 0.0f));
    r[0] = fma2_(splat2(3.0f), d1, fma2_(splat2(-10.0f), d2, mul2_(splat2(13.0f), d3)));
    r[1] = fma2_(splat2(-1.0f), d2, fma2_(splat2(4.0f), d3, mul2_(splat2(3.0f), d4)));
    r[2] = fma2_(splat2(-1.0f), d5, fma2_(splat2(6.0f), d4, d3));
    r[3] = fma2_(splat2(9.0f), d4, fma2_(splat2(-4.0f), d5, d6));
    const float cap = 1.0e15f;
    const float c[4] = {float(K7::C0), float(K7::C1), float(K7::C2), float(K7::C3)};
    const float2 dt = sub2_(is[0], is[3]);
    const float2 tau = make_float2(fabsf(dt.x), fabsf(dt.y));
    float2 al[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float2 q = add2_(splat2(ss), is[k]);
        const float2 t0 = mul2_(tau, make_float2(frcp_fast(q.x), frcp_fast(q.y)));
        const float2 t = make_float2(fminf(t0.x, cap), fminf(t0.y, cap));
        al[k] = mul2_(splat2(c[k]), fma2_(t, t, splat2(1.0f)));
    }
    const float2 num = fma2_(al[3], r[3], fma2_(al[2], r[2], fma2_(al[1], r[1], mul2_(al[0], r[0]))));
    const float2 den = add2_(add2_(add2_(al[0], al[1]), al[2]), al[3]);
    return fma2_(mul2_(num, make_float2(frcp_fast(den.x), frcp_fast(den.y))),
                 splat2(1.0f / 12.0f), f3);
}

// weno3js (weno3js.cpp:79-93 for '+', :134-148 for '-', and its halo
// forms) on an upwind-oriented stencil g0..g2: indicators (g0 - g1)^2 and
// (g1 - g2)^2, candidates -g0/2 + 3 g1/2 and (g1 + g2)/2, linear weights
// 1/3 and 2/3, eps = 1e-6, alpha_k = d_k/(eps + beta_k)^2.  The weights are
// multiplied through by s0^2 s1^2 (s_k = eps + beta_k >= 1e-6, so no product
// leaves the range of either precision), which leaves one reciprocal:
// face = (s1^2 q20 + 2 s0^2 q21) / (s1^2 + 2 s0^2).
template <typename B>
__device__ __forceinline__ B weno3js_face(B g0, B g1, B g2) {
    const B ss = B(1.0e-6);
    const B e0 = sub_(g0, g1), e1 = sub_(g1, g2);
    B s0 = fma_(e0, e0, ss), s1 = fma_(e1, e1, ss);
    s0 = mul_(s0, s0);
    s1 = mul_(s1, s1);
    const B w1 = mul_(B(2), s0);  // (2/3) s0^2 over (1/3) s1^2, times 3
    const B q20 = fma_(B(-0.5), g0, mul_(B(1.5), g1)), q21 = mul_(B(0.5), add_(g1, g2));
    const B den = add_(s1, w1);
    if constexpr (sizeof(B) == 8)
        return mul_(fma_(w1, q21, mul_(s1, q20)), drcp_nr(den));
    else
        return mul_(fma_(w1, q21, mul_(s1, q20)), frcp_fast(den));
}

// ---- hccs77 / hccs78 (hccs77.cpp, hccs78.cpp) ----
// Their WENO7-Z face (eps = 1e-20, squares through pow with their member
// p = 2) and the unnormalised weights' sum S = sum alpha, from which both
// blend with theta = 1/(1 + (S - 1)^2).  FP64 forms S and theta with the
// reference's own operations (a division per weight, x*x for pow(x, 2), the
// sums left to right; the indicators come from weno7_parts in the
// reference's order), so theta, and hccs77's switch on theta > 1/2, come out
// as the reference's.
__device__ __forceinline__ double weno7z_face_sum(double f0, double f1, double f2, double f3,
                                                  double f4, double f5, double f6, double &theta) {
    double is[4], q[4];
    weno7_parts(f0, f1, f2, f3, f4, f5, f6, is, q);
    const double ss = 1.0e-20;
    const double tau = fabs(sub_(is[0], is[3]));
    const double c[4] = {K7::C0, K7::C1, K7::C2, K7::C3};
    double a[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double r = div_(tau, add_(ss, is[k]));
        a[k] = mul_(c[k], add_(1.0, mul_(r, r)));
    }
    const double sa = add_(add_(add_(a[0], a[1]), a[2]), a[3]);
    const double x = sub_(sa, 1.0);
    theta = div_(1.0, add_(1.0, mul_(x, x)));
    const double num = fma_(a[3], q[3], fma_(a[2], q[2], fma_(a[1], q[1], mul_(a[0], q[0]))));
    return div_(num, sa);
}
// FP32 (mixed path): the difference-form WENO7-Z of weno7_face_eps and its
// weights' sum
__device__ __forceinline__ float weno7z_face_sum(float f0, float f1, float f2, float f3, float f4,
                                                 float f5, float f6, float &theta) {
    float d1 = sub_(f1, f0), d2 = sub_(f2, f1), d3 = sub_(f3, f2);
    float d4 = sub_(f4, f3), d5 = sub_(f5, f4), d6 = sub_(f6, f5);
    float s2 = sub_(d2, d1), s3 = sub_(d3, d2), s4 = sub_(d4, d3), s5 = sub_(d5, d4),
          s6 = sub_(d6, d5);
    float is[4], r[4];
    is[0] = w7_beta(d2, s2, s3, -160.0f, 880.0f, 547.0f, -1854.0f, 2107.0f);
    is[1] = w7_beta(d3, s3, s4, 80.0f, 160.0f, 267.0f, -494.0f, 547.0f);
    is[2] = w7_beta(d4, s4, s5, -160.0f, -80.0f, 547.0f, -494.0f, 267.0f);
    is[3] = w7_beta(d5, s5, s6, -880.0f, 160.0f, 2107.0f, -1854.0f, 547.0f);
#pragma unroll
    for (int k = 0; k < 4; ++k) is[k] = fmaxf(is[k], 0.0f);
    r[0] = fma_(3.0f, d1, fma_(-10.0f, d2, mul_(13.0f, d3)));
    r[1] = fma_(-1.0f, d2, fma_(4.0f, d3, mul_(3.0f, d4)));
    r[2] = fma_(-1.0f, d5, fma_(6.0f, d4, d3));
    r[3] = fma_(9.0f, d4, fma_(-4.0f, d5, d6));
    const float ss = 1.0e-20f, cap = 1.0e15f;
    const float c[4] = {float(K7::C0), float(K7::C1), float(K7::C2), float(K7::C3)};
    float tau = fabsf(sub_(is[0], is[3]));
    float al[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float t = fminf(mul_(tau, frcp_fast(add_(ss, is[k]))), cap);
        al[k] = mul_(c[k], fma_(t, t, 1.0f));
    }
    float num = fma_(al[3], r[3], fma_(al[2], r[2], fma_(al[1], r[1], mul_(al[0], r[0]))));
    float den = add_(add_(add_(al[0], al[1]), al[2]), al[3]);
    const float x = sub_(den, 1.0f);
    theta = frcp_fast(fma_(x, x, 1.0f));  // 0 once x^2 overflows
    return fma_(mul_(num, frcp_fast(den)), 1.0f / 12.0f, f3);
}

// hccs78's face on faces 4..n-4 (hccs78.cpp:81-139, '-' :171-229): the
// WENO7-Z face of the upwind-oriented stencil f0..f6 blended with the
// 8th-order central value of the cells c0..c7 around the face (m-4..m+3;
// the same expression for both signs): (1 - theta) W7 + theta q8.
template <typename B>
__device__ __forceinline__ B hccs78_face(B f0, B f1, B f2, B f3, B f4, B f5, B f6, B c0, B c1, B c2,
                                         B c3, B c4, B c5, B c6, B c7) {
    B theta;
    const B w7 = weno7z_face_sum(f0, f1, f2, f3, f4, f5, f6, theta);
    const B q8 = mul_(add_(add_(add_(mul_(B(-3), add_(c7, c0)), mul_(B(29), add_(c6, c1))),
                                mul_(B(-139), add_(c5, c2))),
                           mul_(B(533), add_(c4, c3))),
                      B(1.0 / 840.0));
    return add_(mul_(sub_(B(1), theta), w7), mul_(theta, q8));
}

// One row of hccs77 (hccs77.cpp:79-162 for '+', :246-305 for '-'), from the
// upwind-oriented 7-cell stencil g0..g6 of the row's cell i ('+': cells
// i-3..i+3): theta > 1/2 gives the linear upwind compact row (2/7, 4/7, 1/7
// | q7), otherwise (2/7 theta, 1 - 3/7 theta, 1/7 theta | (1 - theta) W7 +
// theta q7); lo couples the upwind-side face, hi the downwind side.
template <typename B>
__device__ __forceinline__ void h77_row(B g0, B g1, B g2, B g3, B g4, B g5, B g6, B &lo, B &b,
                                        B &hi, B &d) {
    B theta;
    const B w7 = weno7z_face_sum(g0, g1, g2, g3, g4, g5, g6, theta);
    const B q7 = mul_(fma_(B(4), g5, fma_(B(159), g4, fma_(B(239), g3, fma_(B(19), g2, -g1)))),
                      B(1.0 / 420.0));
    if (theta > B(0.5)) {
        lo = B(2.0 / 7.0);
        b = B(4.0 / 7.0);
        hi = B(1.0 / 7.0);
        d = q7;
    } else {
        lo = mul_(B(2.0 / 7.0), theta);
        b = add_(B(1), mul_(B(4.0 / 7.0 - 1.0), theta));
        hi = mul_(B(1.0 / 7.0), theta);
        d = add_(mul_(w7, sub_(B(1), theta)), mul_(q7, theta));
    }
}

// One hybrid row of hccs (hccs.cpp:138-185; '-' mirrored, :375-420), scaled
// by a positive factor.  WENO5-Z-type weights over the CRWENO5 linear
// weights, alpha_k = c_k (1 + (tau/(beta_k + eps))^2), eps = 1e-40; with
// x = sum alpha - 1 the blend is theta = 1/(1 + x^2).  theta > 1/2 (taken, as
// the reference, as 1 + x^2 < 2) gives the linear upwind compact row
// (2/7, 4/7, 1/7 | q7); otherwise the reference row
//   (CRWENO5 row in omega) (1 - theta)/theta + (2/7, 4/7, 1/7 | q7)
// is used multiplied by sum(alpha)/x^2, i.e. (CRWENO5 row in alpha) +
// (2/7, 4/7, 1/7 | q7) sum(alpha)/x^2 (the two factors are equal in exact
// arithmetic; this form stays finite for any x).
//   FP64: the alphas multiplied through by P = s0 s1 s2, s_k = (beta_k +
//   eps)^2 (at least 1e-80 each, so P does not underflow), x = (sum A - P)/P.
//   FP32: reciprocal form with eps = 1e-30 + the stencil's FP32 noise floor
//   and tau/(beta + eps) capped; the weighted row in normalised weights,
//   scaled by 1/x^2.
__device__ __forceinline__ void hc_row(double f0, double f1, double f2, double f3, double f4,
                                       double &lo, double &b, double &hi, double &d) {
    // indicators times 4 (weno5_beta4) with eps alike: every alpha and the
    // products below scale by 16^3, which leaves x and the row's ratios as
    // they are (a row may be scaled freely)
    double is0, is1, is2;
    weno5_beta4(f0, f1, f2, f3, f4, is0, is1, is2);
    const double q7 = mul_(fma_(4.0, f4, fma_(159.0, f3, fma_(239.0, f2, fma_(19.0, f1, -f0)))),
                           1.0 / 420.0);
    const double ss = 4.0 * 1.0e-40;
    const double tau = fabs(sub_(is2, is0));
    const double t2 = mul_(tau, tau);
    double s0 = add_(is0, ss), s1 = add_(is1, ss), s2 = add_(is2, ss);
    s0 = mul_(s0, s0);
    s1 = mul_(s1, s1);
    s2 = mul_(s2, s2);
    // A_k = c_k (s_k + tau^2) prod_{j!=k} s_j = c_k (P + tau^2 prod_{j!=k} s_j)
    const double p12 = mul_(s1, s2), p02 = mul_(s0, s2), p01 = mul_(s0, s1);
    const double P = mul_(s0, p12);
    const double A0 = mul_(K::CR0, fma_(t2, p12, P));
    const double A1 = mul_(K::CR1, fma_(t2, p02, P));
    const double A2 = mul_(K::CR2, fma_(t2, p01, P));
    const double SA = add_(add_(A0, A1), A2);
    // theta = 1/(1 + x^2) > 1/2 with x = sum(alpha) - 1 = (SA - P)/P, i.e.
    // |SA - P| < P: decided without a division
    const double dSP = sub_(SA, P);
    if (fabs(dSP) < P) {
        lo = 2.0 / 7.0;
        b = 4.0 / 7.0;
        hi = 1.0 / 7.0;
        d = q7;
        return;
    }
    const double ix = mul_(P, drcp_nr(dSP));  // 1/x
    const double u = mul_(mul_(SA, ix), ix);            // P sum(alpha) / x^2
    const double third = 1.0 / 3.0, two3 = 2.0 / 3.0, sixth = 1.0 / 6.0;
    lo = fma_(2.0 / 7.0, u, fma_(two3, A0, mul_(third, A1)));
    b = fma_(4.0 / 7.0, u, fma_(third, A0, mul_(two3, add_(A1, A2))));
    hi = fma_(1.0 / 7.0, u, mul_(third, A2));
    d = fma_(q7, u, fma_(mul_(sixth, add_(A1, mul_(5.0, A2))), f3,
                         fma_(mul_(sixth, add_(mul_(5.0, add_(A0, A1)), A2)), f2,
                              mul_(mul_(sixth, A0), f1))));
}
__device__ __forceinline__ void hc_row(float f0, float f1, float f2, float f3, float f4, float &lo,
                                       float &b, float &hi, float &d) {
    // indicators times 4 (weno5_beta4); tau and eps scale alike, so the
    // ratios r_k below are unchanged
    float is0, is1, is2;
    weno5_beta4(f0, f1, f2, f3, f4, is0, is1, is2);
    const float q7 = mul_(fma_(4.0f, f4, fma_(159.0f, f3, fma_(239.0f, f2, fma_(19.0f, f1, -f0)))),
                          float(1.0 / 420.0));
    // eps: the reference's 1e-40 is below FP32's range; in its place the
    // stencil's own FP32 noise floor, (4e-6 max|f|)^2 (a second difference of
    // FP32 values is only known to ~1e-6 of their size).  Indicators below it
    // carry no information: a flat stretch far from the line's offset cell
    // would otherwise get noise-driven, saturated weights, and two saturated
    // neighbouring rows (omega2 = 1, then omega0 = 1) form a singular 2x2
    // block of the line system.  With the floor such stencils take the linear
    // row.
    const float sc = mul_(2.0f * 4.0e-6f, fmaxf(fmaxf(fmaxf(fabsf(f0), fabsf(f1)), fmaxf(fabsf(f2), fabsf(f3))),
                                                fabsf(f4)));
    const float ss = fma_(sc, sc, 4.0f * 1.0e-30f), cap = 1.0e15f;  // 4 (eps + floor^2)
    const float tau = fabsf(sub_(is2, is0));
    const float r0 = fminf(mul_(tau, frcp_fast(add_(is0, ss))), cap);
    const float r1 = fminf(mul_(tau, frcp_fast(add_(is1, ss))), cap);
    const float r2 = fminf(mul_(tau, frcp_fast(add_(is2, ss))), cap);
    const float A0 = mul_(float(K::CR0), fma_(r0, r0, 1.0f));
    const float A1 = mul_(float(K::CR1), fma_(r1, r1, 1.0f));
    const float A2 = mul_(float(K::CR2), fma_(r2, r2, 1.0f));
    const float SA = add_(add_(A0, A1), A2);
    const float x = sub_(SA, 1.0f);
    if (add_(1.0f, mul_(x, x)) < 2.0f) {
        lo = 2.0f / 7.0f;
        b = 4.0f / 7.0f;
        hi = 1.0f / 7.0f;
        d = q7;
        return;
    }
    // FP32 keeps the reference's normalised weights (alphas reach 1e36 here)
    // and scales the row by 1/x^2 (<= 1; 0 if x^2 overflows): every term
    // stays O(1)
    const float is = frcp_fast(SA);
    const float w0 = mul_(A0, is), w1 = mul_(A1, is), w2 = mul_(A2, is);
    const float u = frcp_fast(mul_(x, x));
    const float third = 1.0f / 3.0f, two3 = 2.0f / 3.0f, sixth = 1.0f / 6.0f;
    lo = fma_(2.0f / 7.0f, u, fma_(two3, w0, mul_(third, w1)));
    b = fma_(4.0f / 7.0f, u, fma_(third, w0, mul_(two3, add_(w1, w2))));
    hi = fma_(1.0f / 7.0f, u, mul_(third, w2));
    d = fma_(q7, u, fma_(mul_(sixth, add_(w1, mul_(5.0f, w2))), f3,
                         fma_(mul_(sixth, add_(mul_(5.0f, add_(w0, w1)), w2)), f2,
                              mul_(mul_(sixth, w0), f1))));
}

// CD6 first derivative (centraldifference6th.cpp:44-46), times 1/dx.
template <typename B>
__device__ __forceinline__ B cd6(B m3, B m2, B m1, B p1, B p2, B p3, B inv_dx) {
    return (B(K::CD3) * (p3 - m3) + B(K::CD2) * (p2 - m2) + B(K::CD1) * (p1 - m1)) * inv_dx;
}

// Derivative of a whole-box field f at cell (i, j, k) along axis d with the
// periodic wrap by the direction's differential scheme (centraldifference6th
// .cpp:44-46, centraldifference2nd.cpp:44, centraldifference8th.cpp:120-123
// on one rank), FP64; the diagnostics' gradients (statistics, spectra).
__device__ __forceinline__ double diff_at(const double *f, const BoxParams &p, int i, int j, int k,
                                          int d) {
    const int n = p.n[d];
    const int c = d == 0 ? i : (d == 1 ? j : k);
    const long long base = (long long)i + p.stride[1] * j + p.stride[2] * k - p.stride[d] * c;
    auto at = [&](int o) { return f[base + p.stride[d] * wrap(c + o, n)]; };
    if (p.vis[d] == VIS_CD2) return K::C21 * (at(1) - at(-1)) / p.d[d];
    if (p.vis[d] == VIS_CD8)
        return (K::C84 * (at(4) - at(-4)) + K::C83 * (at(3) - at(-3)) +
                K::C82 * (at(2) - at(-2)) + K::C81 * (at(1) - at(-1))) /
               p.d[d];
    return (K::CD3 * (at(3) - at(-3)) + K::CD2 * (at(2) - at(-2)) + K::CD1 * (at(1) - at(-1))) /
           p.d[d];
}

// Viscosity and heat-conduction coefficient (physicsModel.cpp:193-266).
template <typename B>
__device__ __forceinline__ void viscosity(const BoxParams &bp, B T, B &miu, B &coeff) {
    B m;
    if (bp.visc_model == VISC_SUTHERLAND) {
        B tr = B(bp.tref_nd);
        m = (B(1) + tr) / (T + tr) * (T * sqrt(T)) / B(bp.reynolds);
    } else if (bp.visc_model == VISC_CONSTANT) {
        m = B(1) / B(bp.reynolds);
    } else {
        m = pow(T, B(bp.powerlaw_exp)) / B(bp.reynolds);
    }
    miu = m;
    coeff = m / B((bp.gamma - 1.0) * bp.mach * bp.mach * bp.prandtl);
}

// The same coefficients with the box's constants formed once per block:
// Sutherland as ((1 + Tref)/Re) T sqrt(T) / (T + Tref) with one correctly
// rounded reciprocal, and the divisions by Re and by (gamma-1) M^2 Pr as
// multiplications by their reciprocals (each within an ulp or two of the
// reference's divisions).
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }
template <typename B>
struct ViscConst {
    int model;
    B tr, suth, inv_re, pexp, heat;
    __device__ explicit ViscConst(const BoxParams &bp)
        : model(bp.visc_model),
          tr(B(bp.tref_nd)),
          suth(B((1.0 + bp.tref_nd) / bp.reynolds)),
          inv_re(B(1.0 / bp.reynolds)),
          pexp(B(bp.powerlaw_exp)),
          heat(B(1.0 / ((bp.gamma - 1.0) * bp.mach * bp.mach * bp.prandtl))) {}
    __device__ __forceinline__ void eval(B T, B &miu, B &coeff) const {
        B m;
        if (model == VISC_SUTHERLAND)
            m = suth * (T * sqrt(T)) * rcp_rn(T + tr);
        else if (model == VISC_CONSTANT)
            m = inv_re;
        else
            m = pow(T, pexp) * inv_re;
        miu = m;
        coeff = m * heat;
    }
};

// atomic max of a non-negative double (its bit pattern orders as an integer)
__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long *>(addr),
              static_cast<unsigned long long>(__double_as_longlong(v)));
}

}  // namespace nuc3d
