// Per-operator kernels behind nuc3d_reconstruct / nuc3d_cd6 /
// nuc3d_tvdrk3_stage: the reference's scheme plug-in interface
// (fieldOperator.h:13-81) on device buffers, with explicit halos.
//
// Convention (as the reference): the operator runs along the fastest axis of
// an (nx,ny,nz) field; halo_l / halo_r are (H,ny,nz) arrays holding the H
// cells beyond each end of every line (H = 4 for weno7js, 3 otherwise);
// reconstruction output is (nx+1,ny,nz).
#include "nuc3d_device.cuh"
#include "op_kernels.h"

namespace nuc3d {

namespace {

// value of cell c (-H <= c < nx+H) of line (j,k); the halos are (H,ny,nz)
template <int H = 3>
__device__ __forceinline__ double line_at(const double *in, const double *hl, const double *hr,
                                          int nx, long long line, int c) {
    if (c < 0) return hl[H * line + (c + H)];
    if (c >= nx) return hr[H * line + (c - nx)];
    return in[(long long)nx * line + c];
}

}  // namespace

// One thread per face.  weno5js.cpp:39-628 / weno5z.cpp:38-637: every face m
// reads cells m-3..m+1 ('+') or m+2..m-2 ('-'); faces 3..nx-3 are the
// "inner" faces where weno5z.cpp:80 applies.
template <int SCHEME>
__global__ void k_op_weno(int upwind, unsigned quirks, int nx, long long lines, const double *in,
                          const double *hl, const double *hr, double *out) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long total = (long long)(nx + 1) * lines;
    if (t >= total) return;
    long long line = t / (nx + 1);
    int m = (int)(t - line * (nx + 1));
    double f[5];
#pragma unroll
    for (int k = 0; k < 5; ++k)
        f[k] = upwind > 0 ? line_at(in, hl, hr, nx, line, m - 3 + k)
                          : line_at(in, hl, hr, nx, line, m + 2 - k);
    bool quirk = SCHEME == SCHEME_Z && upwind > 0 && (quirks & QK_WENOZ_BETA2) && m >= 3 &&
                 m <= nx - 3;
    out[t] = SCHEME == SCHEME_Z ? weno5z_face(f[0], f[1], f[2], f[3], f[4], quirk)
                                : weno5js_face(f[0], f[1], f[2], f[3], f[4]);
}

// One thread per face of weno3js (weno3js.cpp:44-483: cells m-2..m for '+',
// m+1..m-1 for '-', 2-cell halos) or upwind1st (upwind1st.cpp:40-368: the
// upwind cell, 1-cell halos).
template <int SCH>
__global__ void k_op_low(int upwind, int nx, long long lines, const double *in, const double *hl,
                         const double *hr, double *out) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long total = (long long)(nx + 1) * lines;
    if (t >= total) return;
    long long line = t / (nx + 1);
    int m = (int)(t - line * (nx + 1));
    constexpr int H = scheme_halo(SCH);
    if (SCH == SCHEME_U1) {
        out[t] = line_at<H>(in, hl, hr, nx, line, upwind > 0 ? m - 1 : m);
        return;
    }
    if (upwind > 0)
        out[t] = weno3js_face(line_at<H>(in, hl, hr, nx, line, m - 2),
                              line_at<H>(in, hl, hr, nx, line, m - 1),
                              line_at<H>(in, hl, hr, nx, line, m));
    else
        out[t] = weno3js_face(line_at<H>(in, hl, hr, nx, line, m + 1),
                              line_at<H>(in, hl, hr, nx, line, m),
                              line_at<H>(in, hl, hr, nx, line, m - 1));
}

// One thread per face of weno7js (weno7js.cpp:17-824) or hccs78
// (hccs78.cpp:44-732): face m reads cells m-4..m+2 ('+') or m+3..m-3 ('-');
// the boundary faces use the same expression on halo cells.  hccs78 blends
// faces 4..nx-4 with the central value of cells m-4..m+3.
template <bool H78>
__global__ void k_op_weno7(int upwind, int nx, long long lines, const double *in,
                           const double *hl, const double *hr, double *out) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long total = (long long)(nx + 1) * lines;
    if (t >= total) return;
    long long line = t / (nx + 1);
    int m = (int)(t - line * (nx + 1));
    double f[7];
#pragma unroll
    for (int k = 0; k < 7; ++k)
        f[k] = upwind > 0 ? line_at<4>(in, hl, hr, nx, line, m - 4 + k)
                          : line_at<4>(in, hl, hr, nx, line, m + 3 - k);
    if (H78 && m >= 4 && m <= nx - 4) {
        double c[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) c[k] = line_at<4>(in, hl, hr, nx, line, m - 4 + k);
        out[t] = hccs78_face(f[0], f[1], f[2], f[3], f[4], f[5], f[6], c[0], c[1], c[2], c[3],
                             c[4], c[5], c[6], c[7]);
        return;
    }
    out[t] = weno7_face(f[0], f[1], f[2], f[3], f[4], f[5], f[6]);
}

// One thread per line: crweno5.cpp:45-402 + halo faces :425-837.  scratch
// holds 2*nx values per line (c' and d' of the Thomas sweep), interleaved
// with the line index fastest (row r of line l at r*lines + l, d' rows after
// the nx c' rows), so that the consecutive lines of a warp touch consecutive
// words.
__global__ void k_op_crweno(int upwind, int nx, long long lines, const double *in,
                            const double *hl, const double *hr, double *out, double *scratch) {
    long long line = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (line >= lines) return;
    auto F = [&](int c) { return line_at(in, hl, hr, nx, line, c); };
    auto js = [&](int m) {
        if (upwind > 0) return weno5js_face(F(m - 3), F(m - 2), F(m - 1), F(m), F(m + 1));
        return weno5js_face(F(m + 2), F(m + 1), F(m), F(m - 1), F(m - 2));
    };
    double *o = out + (long long)(nx + 1) * line;
    for (int m = 0; m <= 2; ++m) o[m] = js(m);
    for (int m = nx - 2; m <= nx; ++m) o[m] = js(m);
    const int M = nx - 5;
    double *cs = scratch + line;                    // c' of row r at cs[r * lines]
    double *ds = scratch + (long long)nx * lines + line;  // d' of row r at ds[r * lines]
    double cp = 0.0, dp = js(3);
    cs[0] = cp;
    ds[0] = dp;
    for (int r = 1; r < M; ++r) {
        double a, b, c, d;
        if (r == M - 1) {
            a = 0.0; b = 1.0; c = 0.0; d = js(r + 3);
        } else {
            int i = r + 2;
            double f0, f1, f2, f3, f4;
            if (upwind > 0) {
                f0 = F(i - 2); f1 = F(i - 1); f2 = F(i); f3 = F(i + 1); f4 = F(i + 2);
            } else {
                f0 = F(i + 3); f1 = F(i + 2); f2 = F(i + 1); f3 = F(i); f4 = F(i - 1);
            }
            double is0, is1, is2;
            weno5_beta(f0, f1, f2, f3, f4, is0, is1, is2, false);
            double a0 = K::CR0 / ((1e-6 + is0) * (1e-6 + is0));
            double a1 = K::CR1 / ((1e-6 + is1) * (1e-6 + is1));
            double a2 = K::CR2 / ((1e-6 + is2) * (1e-6 + is2));
            double sum = a0 + a1 + a2;
            double w0 = a0 / sum, w1 = a1 / sum, w2 = a2 / sum;
            double lo = 2.0 / 3.0 * w0 + 1.0 / 3.0 * w1;
            double hi = 1.0 / 3.0 * w2;
            b = 1.0 / 3.0 * w0 + 2.0 / 3.0 * (w1 + w2);
            d = 1.0 / 6.0 * w0 * f1 + (5.0 * (w0 + w1) + w2) * f2 / 6.0 + (w1 + 5.0 * w2) * f3 / 6.0;
            if (upwind > 0) { a = lo; c = hi; } else { c = lo; a = hi; }
        }
        double den = b - cp * a;
        cp = c / den;
        dp = (d - dp * a) / den;
        cs[r * lines] = cp;
        ds[r * lines] = dp;
    }
    double x = ds[(M - 1) * lines];
    o[nx - 3] = x;
    for (int r = M - 2; r >= 0; --r) {
        x = ds[r * lines] - cs[r * lines] * x;
        o[r + 3] = x;
    }
}

// One thread per line: hccs (hccs.cpp): faces 0..3 and nx-3..nx explicit
// hccs (hccs.cpp) and hccs77 (hccs77.cpp): WENO7 with hccs's eps
// (:538-980) or hccs77's WENO7-Z (:330-818) at the ends, the system of faces
// 4..nx-4 (identity rows at its ends, hybrid rows between; hccs.cpp:54-245
// / :272-471, hccs77.cpp:44-305) by a Thomas sweep.  scratch holds 2*nx
// values per line, interleaved as in k_op_crweno.
template <int SCH>
__global__ void k_op_hccs(int upwind, int nx, long long lines, const double *in,
                          const double *hl, const double *hr, double *out, double *scratch) {
    long long line = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (line >= lines) return;
    auto F = [&](int c) { return line_at<4>(in, hl, hr, nx, line, c); };
    auto w7face = [&](double f0, double f1, double f2, double f3, double f4, double f5,
                      double f6) {
        return SCH == SCHEME_H77 ? weno7_face(f0, f1, f2, f3, f4, f5, f6)
                                 : weno7_face_hc(f0, f1, f2, f3, f4, f5, f6);
    };
    auto w7 = [&](int m) {
        if (upwind > 0)
            return w7face(F(m - 4), F(m - 3), F(m - 2), F(m - 1), F(m), F(m + 1), F(m + 2));
        return w7face(F(m + 3), F(m + 2), F(m + 1), F(m), F(m - 1), F(m - 2), F(m - 3));
    };
    double *o = out + (long long)(nx + 1) * line;
    for (int m = 0; m <= 3; ++m) o[m] = w7(m);
    for (int m = nx - 3; m <= nx; ++m) o[m] = w7(m);
    const int M = nx - 7;
    double *cs = scratch + line;                    // interleaved as in k_op_crweno
    double *ds = scratch + (long long)nx * lines + line;
    double cp = 0.0, dp = w7(4);
    cs[0] = cp;
    ds[0] = dp;
    for (int r = 1; r < M; ++r) {
        double a, b, c, d;
        if (r == M - 1) {
            a = 0.0; b = 1.0; c = 0.0; d = w7(r + 4);
        } else {
            const int i = r + 3;
            double lo, hi;
            if (SCH == SCHEME_H77) {
                if (upwind > 0)
                    h77_row(F(i - 3), F(i - 2), F(i - 1), F(i), F(i + 1), F(i + 2), F(i + 3), lo, b,
                            hi, d);
                else
                    h77_row(F(i + 4), F(i + 3), F(i + 2), F(i + 1), F(i), F(i - 1), F(i - 2), lo, b,
                            hi, d);
            } else if (upwind > 0) {
                hc_row(F(i - 2), F(i - 1), F(i), F(i + 1), F(i + 2), lo, b, hi, d);
            } else {
                hc_row(F(i + 3), F(i + 2), F(i + 1), F(i), F(i - 1), lo, b, hi, d);
            }
            if (upwind > 0) { a = lo; c = hi; } else { c = lo; a = hi; }
        }
        double den = b - cp * a;
        cp = c / den;
        dp = (d - dp * a) / den;
        cs[r * lines] = cp;
        ds[r * lines] = dp;
    }
    double x = ds[(M - 1) * lines];
    o[nx - 4] = x;
    for (int r = M - 2; r >= 0; --r) {
        x = ds[r * lines] - cs[r * lines] * x;
        o[r + 4] = x;
    }
}

// centraldifference6th.cpp:16-186: one thread per cell.
__global__ void k_op_cd6(int nx, long long lines, double inv_dx, const double *in,
                         const double *hl, const double *hr, double *out) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nx * lines) return;
    long long line = t / nx;
    int i = (int)(t - line * nx);
    auto F = [&](int c) { return line_at(in, hl, hr, nx, line, c); };
    out[t] = cd6<double>(F(i - 3), F(i - 2), F(i - 1), F(i + 1), F(i + 2), F(i + 3), inv_dx);
}

// centraldifference2nd.cpp:16-146 / centraldifference8th.cpp:22-205 (and
// centraldifference6th with any tilesize): one thread per cell, halos of the
// tilesize's width.  cd8's cells at least `tile` from both line ends take its
// inner form (the two one-sided sums, :50-60), the others its symmetric
// differences (:120-123, :188-191); cd2 and cd6 have one form.
template <int SCH>
__global__ void k_op_diff(int nx, int tile, long long lines, double dx, const double *in,
                          const double *hl, const double *hr, double *out) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nx * lines) return;
    long long line = t / nx;
    int i = (int)(t - line * nx);
    auto F = [&](int c) {
        if (c < 0) return hl[tile * line + (c + tile)];
        if (c >= nx) return hr[tile * line + (c - nx)];
        return in[(long long)nx * line + c];
    };
    double r;
    if constexpr (SCH == VIS_CD2) {
        r = div_(mul_(K::C21, sub_(F(i + 1), F(i - 1))), dx);
    } else if constexpr (SCH == VIS_CD8) {
        if (i >= tile && i < nx - tile) {
            const double an = add_(add_(add_(mul_(K::C84, F(i - 4)), mul_(K::C83, F(i - 3))),
                                        mul_(K::C82, F(i - 2))),
                                   mul_(K::C81, F(i - 1)));
            const double ap = add_(add_(add_(mul_(K::C81, F(i + 1)), mul_(K::C82, F(i + 2))),
                                        mul_(K::C83, F(i + 3))),
                                   mul_(K::C84, F(i + 4)));
            r = div_(sub_(ap, an), dx);
        } else {
            r = div_(add_(add_(add_(mul_(K::C84, sub_(F(i + 4), F(i - 4))),
                                    mul_(K::C83, sub_(F(i + 3), F(i - 3)))),
                               mul_(K::C82, sub_(F(i + 2), F(i - 2)))),
                          mul_(K::C81, sub_(F(i + 1), F(i - 1)))),
                     dx);
        }
    } else {
        r = div_(add_(add_(mul_(K::CD3, sub_(F(i + 3), F(i - 3))),
                           mul_(K::CD2, sub_(F(i + 2), F(i - 2)))),
                      mul_(K::CD1, sub_(F(i + 1), F(i - 1)))),
                 dx);
    }
    out[t] = r;
}

// TVD-RK3.cpp:76-196
__global__ void k_op_rk3(int stage, long long n, double dt, RK5 rk) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= 5 * n) return;
    int e = (int)(t / n);
    long long i = t - e * n;
    double rhs = -rk.rhs[e][i];
    double u;
    if (stage == 0) {
        u = 1.0 * rk.ui[e][i] + 1.0 * rhs * dt;
    } else if (stage == 1) {
        u = 0.75 * rk.un[e][i] + 0.25 * (rhs * dt + rk.ui[e][i]);
    } else {
        u = (1.0 / 3.0) * rk.un[e][i] + (2.0 / 3.0) * (rhs * dt + rk.ui[e][i]);
    }
    rk.ui[e][i] = u;
}

cudaError_t op_reconstruct(int scheme, int upwind, unsigned quirks, int nx, long long lines,
                           const double *in, const double *hl, const double *hr, double *out,
                           cudaStream_t st) {
    if (scheme == SCHEME_CR || scheme == SCHEME_HC || scheme == SCHEME_H77) {
        double *scratch = nullptr;
        size_t bytes = sizeof(double) * 2 * (size_t)nx * (size_t)lines;
        cudaError_t e = cudaMallocAsync(&scratch, bytes, st);
        if (e != cudaSuccess) return e;
        unsigned grid = (unsigned)((lines + 127) / 128);
        if (scheme == SCHEME_HC)
            k_op_hccs<SCHEME_HC><<<grid, 128, 0, st>>>(upwind, nx, lines, in, hl, hr, out, scratch);
        else if (scheme == SCHEME_H77)
            k_op_hccs<SCHEME_H77><<<grid, 128, 0, st>>>(upwind, nx, lines, in, hl, hr, out, scratch);
        else
            k_op_crweno<<<grid, 128, 0, st>>>(upwind, nx, lines, in, hl, hr, out, scratch);
        e = cudaGetLastError();
        cudaError_t f = cudaFreeAsync(scratch, st);
        return e != cudaSuccess ? e : f;
    }
    long long total = (long long)(nx + 1) * lines;
    unsigned grid = (unsigned)((total + 255) / 256);
    if (scheme == SCHEME_W7)
        k_op_weno7<false><<<grid, 256, 0, st>>>(upwind, nx, lines, in, hl, hr, out);
    else if (scheme == SCHEME_H78)
        k_op_weno7<true><<<grid, 256, 0, st>>>(upwind, nx, lines, in, hl, hr, out);
    else if (scheme == SCHEME_W3)
        k_op_low<SCHEME_W3><<<grid, 256, 0, st>>>(upwind, nx, lines, in, hl, hr, out);
    else if (scheme == SCHEME_U1)
        k_op_low<SCHEME_U1><<<grid, 256, 0, st>>>(upwind, nx, lines, in, hl, hr, out);
    else if (scheme == SCHEME_Z)
        k_op_weno<SCHEME_Z><<<grid, 256, 0, st>>>(upwind, quirks, nx, lines, in, hl, hr, out);
    else
        k_op_weno<SCHEME_JS><<<grid, 256, 0, st>>>(upwind, quirks, nx, lines, in, hl, hr, out);
    return cudaGetLastError();
}

cudaError_t op_crweno_into(int upwind, int nx, long long lines, const double *in,
                           const double *hl, const double *hr, double *out, double *scratch,
                           cudaStream_t st) {
    unsigned grid = (unsigned)((lines + 127) / 128);
    k_op_crweno<<<grid, 128, 0, st>>>(upwind, nx, lines, in, hl, hr, out, scratch);
    return cudaGetLastError();
}

cudaError_t op_cd6(int nx, long long lines, double dx, const double *in, const double *hl,
                   const double *hr, double *out, cudaStream_t st) {
    long long total = (long long)nx * lines;
    k_op_cd6<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(nx, lines, 1.0 / dx, in, hl, hr, out);
    return cudaGetLastError();
}

cudaError_t op_differential(int scheme, int tile, int nx, long long lines, double dx,
                            const double *in, const double *hl, const double *hr, double *out,
                            cudaStream_t st) {
    long long total = (long long)nx * lines;
    const unsigned grid = (unsigned)((total + 255) / 256);
    if (scheme == VIS_CD2)
        k_op_diff<VIS_CD2><<<grid, 256, 0, st>>>(nx, tile, lines, dx, in, hl, hr, out);
    else if (scheme == VIS_CD8)
        k_op_diff<VIS_CD8><<<grid, 256, 0, st>>>(nx, tile, lines, dx, in, hl, hr, out);
    else
        k_op_diff<VIS_CD6><<<grid, 256, 0, st>>>(nx, tile, lines, dx, in, hl, hr, out);
    return cudaGetLastError();
}

cudaError_t op_rk3(int stage, long long n, double dt, RK5 rk, cudaStream_t st) {
    long long total = 5 * n;
    k_op_rk3<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(stage, n, dt, rk);
    return cudaGetLastError();
}

}  // namespace nuc3d
