// CRWENO5 / hccs sweeps along y and z for the reference's bounded lines:
// one thread per (line, sign) system, solved by the reference's own Thomas
// recurrences (crweno5.cpp:208-219, hccs.cpp the same).
//
// Lines along y or z are adjacent in x, so a warp of 16 lines x 2 signs
// (lane 2l: line l's '+' system, lane 2l+1: its '-' system) reads each row
// of its 16 lines as one 128-byte FP64 segment.  Each thread walks its line
// once per equation:
//   forward: a sliding window of 2H split fluxes (its sign, cells m-H ..
//            m+H-1 for face m) gives the explicit faces at both ends (kept in
//            registers) and the rows of faces H .. n-H (identity rows at
//            both ends, compact rows between; crweno5.cpp:136-161 via
//            cr_row, or hccs's hc_row); the Thomas coefficients c', d' of
//            every row go to a line-fastest scratch of the box (16-byte
//            stores, coalesced across the warp);
//   backward: x_r = d'_r - c'_r x_{r+1} from the last row down; the two
//            signs of a line meet by a lane shuffle, F^ = F^+ + F^-, and the
//            '+' lane adds (F^_{m+1} - F^_m) / dy to the RHS of cell m.
// The scratch is 2 signs x (n + 1) rows x 2 coefficients per line of the
// box, allocated with the box.  Periodic lines (not in the reference) keep
// the partitioned solve of crweno_kernels.cu.
#include "nuc3d_device.cuh"
#include "rhs_kernels.h"

namespace nuc3d {

namespace {

constexpr int kThLines = 64;               // lines per block (two threads each)
constexpr int kThThreads = 2 * kThLines;

template <typename B>
struct Pair;
template <>
struct Pair<double> {
    using T = double2;
};
template <>
struct Pair<float> {
    using T = float2;
};

__device__ __forceinline__ double rcp_t(double x) { return drcp_nr(x); }
__device__ __forceinline__ float rcp_t(float x) { return frcp_fast(x); }

}  // namespace

// Work item (box, a, b, -): lines i = a*64 .. a*64+63 (those < nx) at k = b
// (DIR 1) or j = b (DIR 2).
template <typename B, int DIR, int SCH>
__global__ void __launch_bounds__(kThThreads)
    k_cr_thomas(const BoxDev *__restrict__ boxes, const WorkItem *__restrict__ items, int in_slot,
                int accumulate) {
    static_assert(DIR == 1 || DIR == 2, "y and z lines only");
    constexpr int H = scheme_halo(SCH);  // explicit faces per end, first unknown face
    constexpr int WS = 2 * H;            // window: cells m-H .. m+H-1 of face m
    using P2 = typename Pair<B>::T;
    const WorkItem it = items[blockIdx.x];
    const BoxDev &bd = boxes[it.box];
    if (!bd.active) return;
    const BoxParams &bp = bd.p;
    const long long np = bd.np;
    const double *const qbase = fieldU(bd, in_slot, 0);
    const double *const wbase = fieldW(bd, 0);
    B *const rbase = fieldR<B>(bd, 0);
    P2 *const scr = static_cast<P2 *>(bd.line_scratch);
    const int n = bp.n[DIR];
    const int nx = bp.n[0];
    const int fixed = it.b;
    const int li = threadIdx.x >> 1, sg = threadIdx.x & 1;
    const int i = it.a * kThLines + li;
    const bool valid = i < nx;
    const int ic = valid ? i : nx - 1;  // lanes past the box read a real line, write nothing
    const long long sy = bp.stride[1], sz = bp.stride[2];
    auto gidx = [&](int pos) -> long long {
        return DIR == 1 ? ic + sy * pos + sz * fixed : ic + sy * fixed + sz * pos;
    };
    const long long lines = DIR == 1 ? (long long)nx * bp.n[2] : (long long)nx * bp.n[1];
    const long long lg = (long long)ic + (long long)nx * fixed;  // this line's scratch column
    auto sidx = [&](int r) -> long long { return ((long long)r * lines + lg) * 2 + sg; };
    const int riemann = bp.riemann;
    const bool mixed = sizeof(B) == sizeof(float);
    const B inv_d = B(bp.inv_d[DIR]);
    const int N = n - (2 * H - 1);  // unknowns: faces H .. n-H

    for (int e = 0; e < 5; ++e) {
        // this sign's split flux of the cell at pos, FP64 (LF / AUSM / AUSMp,
        // as the staging of the other sweeps)
        auto splitf = [&](int pos) -> double {
            const long long g = gidx(pos);
            const double qe = qbase[e * np + g];
            const double un = wbase[DIR * np + g], p = wbase[3 * np + g], c = wbase[4 * np + g];
            double fp, fm;
            if (riemann == RIEMANN_LF) {  // block-uniform; physicsModel.cpp:546-565
                const double hun = mul_(0.5, un), hlam = mul_(0.5, add_(fabs(un), c));
                double hf;
                if (e == 4)
                    hf = mul_(hun, add_(qe, p));
                else if (e == 1 + DIR)
                    hf = fma_(hun, qe, mul_(0.5, p));
                else
                    hf = mul_(hun, qe);
                fp = fma_(hlam, qe, hf);
                fm = fma_(-hlam, qe, hf);
            } else {
                SplitCell sc;
                split_prepare(riemann, un, p, c, sc);
                split_eq<DIR>(riemann, sc, e, qe, fp, fm);
            }
            return sg == 0 ? fp : fm;
        };
        // mixed precision: the line's value at cell 0 is subtracted before
        // rounding to FP32 (WENO commutes with a constant, which cancels in
        // the face difference)
        const double ref = mixed ? splitf(0) : 0.0;
        auto F = [&](int c) -> B {
            int pos = c < 0 ? c + n : (c >= n ? c - n : c);
            return B(mixed ? sub_(splitf(pos), ref) : splitf(pos));
        };
        B w[WS];
#pragma unroll
        for (int k = 0; k < WS - 1; ++k) w[k] = F(-H + k);
        // The two signs share a warp (alternate lanes), so the sign picks the
        // stencil's cells by selects and every lane runs the same code.
        // Explicit face of this sign from the window (face m: '+' reads cells
        // m-H .. m+H-2, '-' cells m+H-1 .. m-H+1).
        const bool minus = sg != 0;
        auto expl = [&](void) -> B {
            if (SCH == SCHEME_HC) {
                B g[7];
#pragma unroll
                for (int k = 0; k < 7; ++k) g[k] = minus ? w[7 - k] : w[k];
                return weno7_face_hc(g[0], g[1], g[2], g[3], g[4], g[5], g[6]);
            }
            B g[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) g[k] = minus ? w[5 - k] : w[k];
            return weno5js_face(g[0], g[1], g[2], g[3], g[4]);
        };
        B xs[H], xe[H];  // explicit faces 0 .. H-1 and n-H+1 .. n
        B cprev = B(0), dprev = B(0);
        for (int m = 0; m <= n; ++m) {
            w[WS - 1] = F(m + H - 1);
            if (m < H) {
                xs[m] = expl();
            } else if (m > n - H) {
                xe[m - (n - H + 1)] = expl();
            } else {
                const int r = m - H;
                B a, b, c, d;
                if (r == 0 || r == N - 1) {  // identity rows hold the explicit faces
                    a = B(0);
                    b = B(1);
                    c = B(0);
                    d = expl();
                } else {
                    // the compact row of cell m-1: '+' reads cells m-3 .. m+1,
                    // '-' cells m+2 .. m-2 with lo and hi swapped
                    // (crweno5.cpp:335-338)
                    B g[5], lo, hi;
#pragma unroll
                    for (int k = 0; k < 5; ++k) g[k] = minus ? w[H + 2 - k] : w[H - 3 + k];
                    if (SCH == SCHEME_HC)
                        hc_row(g[0], g[1], g[2], g[3], g[4], lo, b, hi, d);
                    else
                        cr_row(g[0], g[1], g[2], g[3], g[4], lo, b, hi, d);
                    a = minus ? hi : lo;
                    c = minus ? lo : hi;
                }
                // Thomas forward step (crweno5.cpp:208-214)
                const B rr = rcp_t(b - a * cprev);
                const B cp = c * rr, dp = (d - a * dprev) * rr;
                cprev = cp;
                dprev = dp;
                if (valid) {
                    P2 v;
                    v.x = cp;
                    v.y = dp;
                    scr[sidx(r)] = v;
                }
            }
#pragma unroll
            for (int k = 0; k < WS - 1; ++k) w[k] = w[k + 1];
        }
        // backward (crweno5.cpp:215-219) from face n down to face 0, the two
        // signs of each face added by a shuffle, dF of cell m = (F^_{m+1} - F^_m) / d
        B x = dprev;  // face n-H: the last row
        B fh_next = B(0);
        for (int m = n; m >= 0; --m) {
            B xo;
            if (m > n - H) {
                xo = xe[m - (n - H + 1)];
            } else if (m < H) {
                xo = xs[m];
            } else {
                const int r = m - H;
                if (r < N - 1) {
                    const P2 v = valid ? scr[sidx(r)] : P2{};
                    x = v.y - v.x * x;
                }
                xo = x;
            }
            const B other = __shfl_xor_sync(0xffffffffu, xo, 1);
            const B fh = sg == 0 ? add_(xo, other) : add_(other, xo);  // F^+ + F^-
            if (m < n && sg == 0 && valid) {
                const long long g = gidx(m) + (long long)e * np;
                const B dfe = mul_(sub_(fh_next, fh), inv_d);
                rbase[g] = accumulate ? add_(rbase[g], dfe) : dfe;
            }
            fh_next = fh;
        }
    }
}

template <typename B, int SCH>
static void launch_th(int dir, const BoxDev *boxes, const WorkItem *items, int nitems, int in_slot,
                      int accumulate, cudaStream_t st) {
    if (dir == 1)
        k_cr_thomas<B, 1, SCH><<<nitems, kThThreads, 0, st>>>(boxes, items, in_slot, accumulate);
    else
        k_cr_thomas<B, 2, SCH><<<nitems, kThThreads, 0, st>>>(boxes, items, in_slot, accumulate);
}

int crweno_thomas_lines() { return kThLines; }

size_t crweno_thomas_scratch_bytes(const BoxParams &p, bool mixed) {
    const size_t bs = mixed ? sizeof(float) : sizeof(double);
    const size_t ly = (size_t)p.n[0] * p.n[2] * (p.n[1] + 1);
    const size_t lz = (size_t)p.n[0] * p.n[1] * (p.n[2] + 1);
    return 2 * 2 * bs * (ly > lz ? ly : lz);  // 2 signs x (c', d')
}

template <typename B>
cudaError_t launch_cr_thomas(int sch, int dir, const BoxDev *boxes, const WorkItem *items,
                             int nitems, int in_slot, int accumulate, cudaStream_t st) {
    if (nitems <= 0) return cudaSuccess;
    if (dir != 1 && dir != 2) return cudaErrorInvalidValue;
    if (sch == SCHEME_HC)
        launch_th<B, SCHEME_HC>(dir, boxes, items, nitems, in_slot, accumulate, st);
    else
        launch_th<B, SCHEME_CR>(dir, boxes, items, nitems, in_slot, accumulate, st);
    return cudaGetLastError();
}

template cudaError_t launch_cr_thomas<double>(int, int, const BoxDev *, const WorkItem *, int, int,
                                              int, cudaStream_t);
template cudaError_t launch_cr_thomas<float>(int, int, const BoxDev *, const WorkItem *, int, int,
                                             int, cudaStream_t);

}  // namespace nuc3d
