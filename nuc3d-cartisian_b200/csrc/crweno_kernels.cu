// CRWENO5 whole-box sweep: one thread per (line, equation) solves that
// line's tridiagonal systems for F^+ and F^- and writes dF/dx.
//
// Reference system (crweno5.cpp:45-402, quirk bit QK_CRWENO_BOUNDED set): on
// a line of n cells, faces 0..2 and n-2..n take explicit WENO5-JS values
// from the halo (crweno5.cpp:425-837); faces 3..n-3 solve a tridiagonal
// system whose first and last rows are identity rows holding WENO5-JS values
// and whose inner rows are the compact-WENO relation
//   a F^_{i} + b F^_{i+1} + c F^_{i+2} = d   (row of cell i, face i+1)
// by the Thomas sweep of crweno5.cpp:208-219.
//
// Periodic system (bit cleared; not in the reference): every face 0..n-1 is
// a compact row and the system wraps around; it is solved by Sherman-Morrison
// on top of the same Thomas sweep.
//
// Forward-sweep coefficients and the F^+ face values go to a scratch buffer
// laid out [slot][row][thread] so a warp's accesses are contiguous.
#include "nuc3d_device.cuh"
#include "rhs_kernels.h"

namespace nuc3d {

namespace {

// One compact-WENO row from the upwind-oriented stencil f0..f4 of its cell
// (crweno5.cpp:136-161): returns the upwind-side coupling lo, the diagonal b,
// the downwind-side coupling hi and the right-hand side d.
template <typename B>
__device__ __forceinline__ void crweno_row(B f0, B f1, B f2, B f3, B f4, B &lo, B &b, B &hi,
                                           B &d) {
    B is0, is1, is2;
    weno5_beta(f0, f1, f2, f3, f4, is0, is1, is2, false);
    const B ss = B(1.0e-6);
    B r0 = B(1) / (ss + is0), r1 = B(1) / (ss + is1), r2 = B(1) / (ss + is2);
    B a0 = B(K::CR0) * r0 * r0, a1 = B(K::CR1) * r1 * r1, a2 = B(K::CR2) * r2 * r2;
    B inv = B(1) / (a0 + a1 + a2);
    B w0 = a0 * inv, w1 = a1 * inv, w2 = a2 * inv;
    lo = B(2.0 / 3.0) * w0 + B(1.0 / 3.0) * w1;
    b = B(1.0 / 3.0) * w0 + B(2.0 / 3.0) * (w1 + w2);
    hi = B(1.0 / 3.0) * w2;
    d = B(1.0 / 6.0) * w0 * f1 + (B(5) * (w0 + w1) + w2) * f2 / B(6) + (w1 + B(5) * w2) * f3 / B(6);
}

template <int DIR>
struct LineMap {
    // line id -> base index; positions advance by bp.stride[DIR]
    __device__ static long long base(const BoxParams &bp, long long L) {
        if (DIR == 0) return L * bp.n[0];  // (j,k) rows are contiguous blocks of nx
        if (DIR == 1) {
            long long i = L % bp.n[0], k = L / bp.n[0];
            return i + bp.stride[2] * k;
        }
        return L;  // (i,j): base = i + nx*j = L
    }
    __device__ static long long count(const BoxParams &bp) {
        if (DIR == 0) return (long long)bp.n[1] * bp.n[2];
        if (DIR == 1) return (long long)bp.n[0] * bp.n[2];
        return (long long)bp.n[0] * bp.n[1];
    }
};

}  // namespace

template <typename B, int DIR>
__global__ void __launch_bounds__(128)
    k_crweno(BoxParams bp, StateView q, PrimView w, BView<B> r, int accumulate, B *scratch,
             long long line0, long long chunk, int periodic) {
    const long long T = 5 * chunk;  // threads in this launch
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= T) return;
    const int e = (int)(t / chunk);
    const long long L = line0 + (t - (long long)e * chunk);
    if (L >= LineMap<DIR>::count(bp)) return;
    const int n = bp.n[DIR];
    const long long s = bp.stride[DIR];
    const long long base = LineMap<DIR>::base(bp, L);
    const bool mixed = sizeof(B) == sizeof(float);

    // split flux F^+ (sg=+1) or F^- (sg=-1) of equation e at periodic cell c
    auto fsplit = [&](int c, int sg) -> double {
        c = ((c % n) + n) % n;
        long long g = base + s * c;
        double Qe = q.q[e][g];
        double un = w.w[DIR][g], p = w.w[3][g], cs = w.w[4][g];
        double lam = fabs(un) + cs;
        double f = (e == 4) ? un * (Qe + p) : (e == 1 + DIR ? un * Qe + p : un * Qe);
        return sg > 0 ? 0.5 * (f + lam * Qe) : 0.5 * (f - lam * Qe);
    };
    double ref[2] = {0.0, 0.0};
    if (mixed) {
        ref[0] = fsplit(0, 1);
        ref[1] = fsplit(0, -1);
    }
    auto fb = [&](int c, int sg) -> B { return B(fsplit(c, sg) - ref[sg > 0 ? 0 : 1]); };
    // explicit WENO5-JS face (upwind-oriented stencil)
    auto js = [&](int m, int sg) -> B {
        if (sg > 0) return weno5js_face(fb(m - 3, 1), fb(m - 2, 1), fb(m - 1, 1), fb(m, 1), fb(m + 1, 1));
        return weno5js_face(fb(m + 2, -1), fb(m + 1, -1), fb(m, -1), fb(m - 1, -1), fb(m - 2, -1));
    };
    B *sc_c = scratch;                         // c' per row
    B *sc_d = scratch + (size_t)(n + 1) * T;   // d' per row
    B *sc_h = scratch + 2 * (size_t)(n + 1) * T;  // F^+ per face
    B *sc_z = scratch + 3 * (size_t)(n + 1) * T;  // Sherman-Morrison second solve (periodic)
    auto at = [&](B *slot, int row) -> B & { return slot[(size_t)row * T + t]; };

    const B inv_d = B(bp.inv_d[DIR]);
    B prev = B(0);  // F^ at face m+1 while walking down
    for (int sgi = 0; sgi < 2; ++sgi) {
        const int sg = sgi == 0 ? 1 : -1;
        // row coefficients for cell i (row of face i+1)
        auto row = [&](int i, B &a, B &b, B &c, B &d) {
            B lo, hi;
            if (sg > 0) {
                crweno_row(fb(i - 2, 1), fb(i - 1, 1), fb(i, 1), fb(i + 1, 1), fb(i + 2, 1), lo, b, hi, d);
                a = lo;  // couples face i   (crweno5.cpp:156)
                c = hi;  // couples face i+2
            } else {
                crweno_row(fb(i + 3, -1), fb(i + 2, -1), fb(i + 1, -1), fb(i, -1), fb(i - 1, -1), lo, b, hi, d);
                c = lo;  // crweno5.cpp:335
                a = hi;  // crweno5.cpp:337
            }
        };
        // out(face) consumer: '+' stores, '-' combines and differentiates
        auto emit = [&](int m, B v) {
            if (sg > 0) {
                at(sc_h, m) = v;
            } else {
                B fh = at(sc_h, m) + v;
                if (m < n) {
                    long long g = base + s * m;
                    B dfe = (prev - fh) * inv_d;
                    if (accumulate)
                        r.f[e][g] += dfe;
                    else
                        r.f[e][g] = dfe;
                }
                prev = fh;
            }
        };
        if (!periodic) {
            const int M = n - 5;  // rows for cells 2..n-4 (faces 3..n-3)
            // forward sweep (crweno5.cpp:208-212); row 0 is an identity row
            B cp = B(0), dp = js(3, sg);
            at(sc_c, 0) = cp;
            at(sc_d, 0) = dp;
            for (int rr = 1; rr < M; ++rr) {
                B a, b, c, d;
                if (rr == M - 1) {
                    a = B(0); b = B(1); c = B(0); d = js(rr + 3, sg);
                } else {
                    row(rr + 2, a, b, c, d);
                }
                B den = b - cp * a;
                cp = c / den;
                dp = (d - dp * a) / den;
                at(sc_c, rr) = cp;
                at(sc_d, rr) = dp;
            }
            // walk faces n .. 0
            for (int m = n; m >= n - 2; --m) emit(m, js(m, sg));
            B x = at(sc_d, M - 1);
            emit(n - 3, x);
            for (int rr = M - 2; rr >= 0; --rr) {
                x = at(sc_d, rr) - at(sc_c, rr) * x;
                emit(rr + 3, x);
            }
            for (int m = 2; m >= 0; --m) emit(m, js(m, sg));
        } else {
            // cyclic rows for faces 0..n-1: row of face m belongs to cell m-1.
            // Sherman-Morrison: A = T + u v^T with corner terms moved into u,v.
            B a0, b0, c0, d0, an, bn, cn, dn;
            row(-1, a0, b0, c0, d0);       // face 0
            row(n - 2, an, bn, cn, dn);    // face n-1
            const B gam = -b0;
            // forward sweep for rhs d and rhs u = (gam, 0..0, cn) together
            B cp, dp, zp;
            {
                B bb = b0 - gam;
                cp = c0 / bb;
                dp = d0 / bb;
                zp = gam / bb;
                at(sc_c, 0) = cp;
                at(sc_d, 0) = dp;
                at(sc_z, 0) = zp;
            }
            for (int m = 1; m < n; ++m) {
                B a, b, c, d;
                if (m == n - 1) {
                    a = an; b = bn - a0 * cn / gam; c = cn; d = dn;
                } else {
                    row(m - 1, a, b, c, d);
                }
                B den = b - a * cp;
                B u = (m == n - 1) ? cn : B(0);
                cp = c / den;
                dp = (d - a * dp) / den;
                zp = (u - a * zp) / den;
                at(sc_c, m) = cp;
                at(sc_d, m) = dp;
                at(sc_z, m) = zp;
            }
            // back substitution of both solves; keep x0, z0, x_{n-1}, z_{n-1}
            B x = dp, z = zp;
            at(sc_d, n - 1) = x;
            at(sc_z, n - 1) = z;
            for (int m = n - 2; m >= 0; --m) {
                B cpm = at(sc_c, m);
                x = at(sc_d, m) - cpm * x;
                z = at(sc_z, m) - cpm * z;
                at(sc_d, m) = x;
                at(sc_z, m) = z;
            }
            B xl = at(sc_d, n - 1), zl = at(sc_z, n - 1);
            B fact = (x + a0 * xl / gam) / (B(1) + z + a0 * zl / gam);
            emit(n, at(sc_d, 0) - fact * at(sc_z, 0));  // face n == face 0
            for (int m = n - 1; m >= 0; --m) emit(m, at(sc_d, m) - fact * at(sc_z, m));
        }
    }
}

size_t crweno_scratch_elems(const BoxParams &bp) {
    // 4 slots x (n+1) rows x threads-per-chunk; chunk sized to keep the
    // scratch near L2-resident (~64 MiB of FP64)
    int nmax = bp.n[0] > bp.n[1] ? bp.n[0] : bp.n[1];
    nmax = nmax > bp.n[2] ? nmax : bp.n[2];
    long long per_thread = 4LL * (nmax + 1);
    long long threads = (64LL << 20) / 8 / per_thread;
    if (threads < 5 * 128) threads = 5 * 128;
    return (size_t)(per_thread * threads);
}

template <typename B>
cudaError_t launch_crweno(const BoxParams &bp, int dir, StateView q, PrimView w, BView<B> r,
                          int accumulate, B *scratch, cudaStream_t st, int *nlaunch) {
    int n = bp.n[dir];
    *nlaunch = 0;
    if (n < 8) return cudaErrorInvalidValue;
    int nmax = bp.n[0] > bp.n[1] ? bp.n[0] : bp.n[1];
    nmax = nmax > bp.n[2] ? nmax : bp.n[2];
    long long per_thread = 4LL * (nmax + 1);
    long long threads = (long long)crweno_scratch_elems(bp) / per_thread;
    long long chunk = threads / 5;
    long long lines = dir == 0 ? (long long)bp.n[1] * bp.n[2]
                               : (dir == 1 ? (long long)bp.n[0] * bp.n[2] : (long long)bp.n[0] * bp.n[1]);
    if (chunk > lines) chunk = lines;
    int periodic = (bp.quirks & QK_CRWENO_BOUNDED) ? 0 : 1;
    for (long long l0 = 0; l0 < lines; l0 += chunk) {
        long long T = 5 * chunk;
        unsigned grid = (unsigned)((T + 127) / 128);
        if (dir == 0)
            k_crweno<B, 0><<<grid, 128, 0, st>>>(bp, q, w, r, accumulate, scratch, l0, chunk, periodic);
        else if (dir == 1)
            k_crweno<B, 1><<<grid, 128, 0, st>>>(bp, q, w, r, accumulate, scratch, l0, chunk, periodic);
        else
            k_crweno<B, 2><<<grid, 128, 0, st>>>(bp, q, w, r, accumulate, scratch, l0, chunk, periodic);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return err;
        ++*nlaunch;
    }
    return cudaSuccess;
}

template cudaError_t launch_crweno<double>(const BoxParams &, int, StateView, PrimView,
                                           BView<double>, int, double *, cudaStream_t, int *);
template cudaError_t launch_crweno<float>(const BoxParams &, int, StateView, PrimView,
                                          BView<float>, int, float *, cudaStream_t, int *);

}  // namespace nuc3d
