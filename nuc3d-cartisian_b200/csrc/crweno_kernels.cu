// CRWENO5, hccs and hccs77 directional sweeps, batched over boxes: one block
// per tile of kCrTL lines of one box, one warp per (line, sign) tridiagonal
// system.  hccs (hccs.cpp) has the same bounded structure with 4-cell ends:
// faces 0..3 and n-3..n explicit WENO7 (eps 1e-40), identity rows at faces 4
// and n-4, hybrid compact rows in between (hc_row).  hccs77 (hccs77.cpp)
// has that structure too, with WENO7-Z (eps 1e-20) at the ends and rows that
// blend WENO7-Z into the 7th-order upwind compact row (h77_row).
//
// Reference system (crweno5.cpp:45-402, quirk bit QK_CRWENO_BOUNDED set): on
// a line of n cells, faces 0..2 and n-2..n take explicit WENO5-JS values
// from the halo (crweno5.cpp:425-837); faces 3..n-3 solve a tridiagonal
// system whose first and last rows are identity rows holding WENO5-JS values
// and whose inner rows are the compact-WENO relation of cell i (face i+1)
//   lo F^_i + b F^_{i+1} + hi F^_{i+2} = d          (crweno5.cpp:136-161)
// ('-' swaps lo and hi, crweno5.cpp:335-338).  The reference solves it with
// a Thomas sweep (crweno5.cpp:208-219).
// Periodic system (bit cleared; not in the reference): every face 0..n-1 is
// a compact row and the system wraps around (cyclic tridiagonal).
//
// Per block and equation: the split fluxes F+ and F- of the tile's lines
// (3-cell periodic halo) are staged in shared memory; each warp solves
// one (line, sign) system by a partitioned method — lane l eliminates the
// interior rows of its segment so that every row depends only on the
// segment's first and last unknowns (rows kept at unit diagonal), the 2P
// segment-end unknowns form a tridiagonal (cyclic for periodic lines) system
// that the warp solves by parallel cyclic reduction with shuffles, and
// each lane back-substitutes its interior rows.  The compact rows are used
// without normalising the weights (a row may be scaled freely), so a row
// costs one reciprocal.  The face values overwrite the staged fluxes, and
// the block writes dF/dx.
#include <type_traits>

#include "nuc3d_device.cuh"
#include "prim_device.cuh"
#include "rhs_kernels.h"

namespace nuc3d {

namespace {

constexpr int kCrTL = 4;         // lines per block
constexpr int kCrWarps = 2 * kCrTL;  // one warp per (line, sign) system
constexpr int kCrThreads = 32 * kCrWarps;
constexpr int kCrLanes = 32;          // lanes per system

// CRWENO5 weights up to a common positive factor (crweno5.cpp:136-150:
// alpha_k = c_k / (eps + beta_k)^2, eps = 1e-6, c = 0.2, 0.5, 0.3 = 0.1 (2, 5,
// 3)).  A compact row is linear in the weights and may be scaled freely, so
// the normalisation by their sum is left out and the linear weights go into
// the row's constants (cr_row): cr_p returns p_k with alpha_k proportional to
// c_k p_k.  FP64 multiplies through by the product of the squares (no
// division at all): p_k = prod_{j != k} (eps + beta_j)^2; FP32 uses fast
// reciprocals: p_k = 1 / (eps + beta_k)^2.  The indicators arrive times 4
// (is_k = 4 beta_k) and eps with them, an exact scaling.
__device__ __forceinline__ void cr_p(double is0, double is1, double is2, double &p0, double &p1,
                                     double &p2) {
    const double ss = 4.0 * 1.0e-6;
    double s0 = add_(ss, is0), s1 = add_(ss, is1), s2 = add_(ss, is2);
    s0 = mul_(s0, s0);
    s1 = mul_(s1, s1);
    s2 = mul_(s2, s2);
    p0 = mul_(s1, s2);
    p1 = mul_(s0, s2);
    p2 = mul_(s0, s1);
}
__device__ __forceinline__ void cr_p(float is0, float is1, float is2, float &p0, float &p1,
                                     float &p2) {
    const float ss = 4.0f * 1.0e-6f;
    const float r0 = frcp_fast(add_(ss, is0)), r1 = frcp_fast(add_(ss, is1)),
                r2 = frcp_fast(add_(ss, is2));
    p0 = mul_(r0, r0);
    p1 = mul_(r1, r1);
    p2 = mul_(r2, r2);
}

// One compact-WENO row from the upwind-oriented stencil f0..f4 of its cell:
// the upwind-side coupling lo, the diagonal b, the downwind-side coupling hi
// and the right-hand side d (crweno5.cpp:151-161), all times 60 / (0.1 sum p)
// (a row may be scaled freely): with w = 0.1 (2 p0, 5 p1, 3 p2),
//   lo = 2/3 w0 + 1/3 w1            -> 8 p0 + 10 p1
//   b  = 1/3 w0 + 2/3 (w1 + w2)     -> 4 p0 + 20 p1 + 12 p2
//   hi = 1/3 w2                     -> 6 p2
//   d  = w0/6 f1 + (5 (w0 + w1) + w2)/6 f2 + (w1 + 5 w2)/6 f3
//                                   -> 2 p0 f1 + (10 p0 + 25 p1 + 3 p2) f2 + (5 p1 + 15 p2) f3
template <typename B>
__device__ __forceinline__ void cr_row(B f0, B f1, B f2, B f3, B f4, B &lo, B &b, B &hi, B &d) {
    B is0, is1, is2, p0, p1, p2;
    weno5_beta4(f0, f1, f2, f3, f4, is0, is1, is2);
    cr_p(is0, is1, is2, p0, p1, p2);
    lo = fma_(B(8), p0, mul_(B(10), p1));
    b = fma_(B(4), p0, fma_(B(20), p1, mul_(B(12), p2)));
    hi = mul_(B(6), p2);
    d = fma_(fma_(B(15), p2, mul_(B(5), p1)), f3,
             fma_(fma_(B(10), p0, fma_(B(25), p1, mul_(B(3), p2))), f2, mul_(mul_(B(2), p0), f1)));
}

__device__ __forceinline__ double rcp_(double x) { return drcp_nr(x); }
__device__ __forceinline__ float rcp_(float x) { return frcp_fast(x); }

template <typename B>
__device__ __forceinline__ B shfl(B v, int src) {
    return __shfl_sync(0xffffffffu, v, src);
}

// PCR update of a unit-diagonal row (a, 1, c | d) with its unit-diagonal
// neighbours m (row i - s) and p (row i + s); the result is normalised again.
template <typename B>
__device__ __forceinline__ void pcr_update(B &a, B &c, B &d, B ma, B mc, B md, B pa, B pc, B pd) {
    const B r = rcp_(B(1) - a * mc - c * pa);
    const B nd = (d - a * md - c * pd) * r;
    a = -a * ma * r;
    c = -c * pc * r;
    d = nd;
}

}  // namespace

// unknowns of a line system: bounded lines solve faces H..n-H (the first and
// last as identity rows), periodic ones faces 0..n-1
static int line_unknowns(int sch, int n, bool bounded) {
    const int H = scheme_halo(sch);
    return bounded ? n - (2 * H - 1) : n;
}

int crweno_lanes(int sch, int n, bool bounded) {
    const int N = line_unknowns(sch, n, bounded);
    int P = 1;
    while (P < kCrLanes && 2 * P <= N / 2) P *= 2;
    return P;
}

int crweno_segment_rows(int sch, int n, bool bounded) {
    const int N = line_unknowns(sch, n, bounded);
    const int P = crweno_lanes(sch, n, bounded);
    return (N + P - 1) / P;
}

size_t crweno_smem_bytes(int sch, int nmax, int ms, bool mixed) {
    const size_t bs = mixed ? sizeof(float) : sizeof(double);
    const int H = scheme_halo(sch);
    return bs * ((size_t)2 * kCrTL * (nmax + 2 * H) + (size_t)kCrWarps * 3 * ms * 32);
}

int crweno_tile_lines() { return kCrTL; }

// Work item (box, a, b, -): DIR 0: lines j = a*TL.., k = b; DIR 1: lines
// i = a*TL.., k = b; DIR 2: lines i = a*TL.., j = b.
// prim_mode (x lines only, whose blocks own whole lines): 0 reads the
// primitives W; 1 first recovers the primitives of the block's lines from
// the state (prim_cell, k_prim's work, bitwise the same) and writes W; 2
// also folds their eigenvalues into the box's running maxima.
template <typename B, int DIR, int SCH>
__global__ void __launch_bounds__(kCrThreads, sizeof(B) == 8 ? 3 : 4)
    k_crweno_lines(const BoxDev *__restrict__ boxes, const WorkItem *__restrict__ items,
                   int in_slot, int accumulate, int nmax, int ms, int prim_mode) {
    // SCH: SCHEME_CR (crweno5), SCHEME_HC (hccs) or SCHEME_H77 (hccs77).  H:
    // staged halo, explicit
    // faces per end and the first unknown face (3 for crweno5, 4 for hccs).
    constexpr int H = scheme_halo(SCH);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ls = nmax + 2 * H;                       // staged cells per line
    B *sF = reinterpret_cast<B *>(smem_raw);           // [sign][line][ls]
    B *sRow = sF + 2 * kCrTL * ls;                     // [warp][3][ms][32]
    __shared__ double sRef[2][5][kCrTL];

    const WorkItem it = items[blockIdx.x];
    const BoxDev &bd = boxes[it.box];
    if (!bd.active) return;
    const BoxParams &bp = bd.p;
    const double *const qbase = fieldU(bd, in_slot, 0);
    const double *const wbase = fieldW(bd, 0);
    B *const rbase = fieldR<B>(bd, 0);
    const long long np = bd.np;
    const int n = bp.n[DIR];
    const int l0 = it.a * kCrTL, fixed = it.b;
    const int nl = DIR == 0 ? bp.n[1] : bp.n[0];
    const long long sy = bp.stride[1], sz = bp.stride[2];
    auto gidx = [&](int l, int pos) -> long long {
        const int a = l0 + l;
        if (DIR == 0) return pos + sy * a + sz * fixed;
        if (DIR == 1) return a + sy * pos + sz * fixed;
        return a + sy * fixed + sz * pos;
    };
    // the box's point-wise split (LF / AUSM / AUSMp) of equation e at cell g
    const int riemann = bp.riemann;
    // (the cell's q_e, u_n, p, c already loaded)
    auto split_v = [&](int e, double qe, double un, double p, double c, double &fp, double &fm) {
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
    };
    auto split = [&](int e, long long g, double &fp, double &fm) {
        split_v(e, qbase[e * np + g], wbase[DIR * np + g], wbase[3 * np + g], wbase[4 * np + g],
                fp, fm);
    };
    const bool mixed = sizeof(B) == sizeof(float);
    // hccs lines are always bounded (the reference's form); crweno5 has the
    // periodic form when the quirk bit is cleared
    const bool bounded = SCH != SCHEME_CR || (bp.quirks & QK_CRWENO_BOUNDED) != 0;
    const int N = bounded ? n - (2 * H - 1) : n;  // unknowns of the system
    int P = 1;  // lanes per system
    while (P < kCrLanes && 2 * P <= N / 2) P *= 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // warp w solves line w/2 of the tile for sign w%2 (0: +, 1: -)
    const int line = warp >> 1, sg = warp & 1, hl = lane;
    B *const myF = sF + (sg * kCrTL + line) * ls;  // cell c at [c + H]; later face m at [m]
    B *const wA = sRow + (size_t)warp * 3 * ms * 32;  // [j][lane]
    B *const wC = wA + ms * 32;
    B *const wD = wC + ms * 32;
    const B inv_d = B(bp.inv_d[DIR]);

    if (DIR == 0 && prim_mode != 0) {  // block-uniform
        // con2prim of the block's whole lines: the staging below reads their
        // W (written by this block, visible after the barrier)
        const PrimConst pk(bp);
        double lx = 0.0, ly = 0.0, lz = 0.0;
        // (line, cell) of t = tid, tid + kCrThreads, ... advanced without a division
        int l = threadIdx.x / n, i = threadIdx.x - l * n;
        for (int t = threadIdx.x; t < kCrTL * n; t += kCrThreads) {
            if (t != (int)threadIdx.x) {
                i += kCrThreads;
                while (i >= n) {
                    i -= n;
                    ++l;
                }
            }
            if (l0 + l >= nl) break;  // lines are in order: the rest are outside too
            const long long g = gidx(l, i);
            double Q[5];
#pragma unroll
            for (int q = 0; q < 5; ++q) Q[q] = qbase[q * np + g];
            PrimCell o;
            prim_cell(pk, Q, o);
            prim_store(bd, g, o);
            lx = fmax(add_(fabs(o.u), o.c), lx);
            ly = fmax(add_(fabs(o.v), o.c), ly);
            lz = fmax(add_(fabs(o.w), o.c), lz);
        }
        if (prim_mode == 2) eig_block_max(bd, lx, ly, lz);
        __syncthreads();
    }

    if (mixed) {  // per-line references of the five equations: the split fluxes at cell 0
        if (threadIdx.x < kCrTL) {
            const bool in = l0 + (int)threadIdx.x < nl;
            const long long g = in ? gidx(threadIdx.x, 0) : 0;
            const double un = in ? wbase[DIR * np + g] : 0.0, p = in ? wbase[3 * np + g] : 0.0,
                         c = in ? wbase[4 * np + g] : 0.0;
#pragma unroll
            for (int e = 0; e < 5; ++e) {
                double fp = 0.0, fm = 0.0;
                if (in) split_v(e, qbase[e * np + g], un, p, c, fp, fm);
                sRef[0][e][threadIdx.x] = fp;
                sRef[1][e][threadIdx.x] = fm;
            }
        }
        __syncthreads();
    }
    for (int e = 0; e < 5; ++e) {
        // stage F+ / F- of cells -H .. n+H-1
        const int nst = n + 2 * H;
        // x lines: (line, cell) of t advanced without a division
        int sl = DIR == 0 ? (int)threadIdx.x / nst : 0;
        int spc = DIR == 0 ? (int)threadIdx.x - sl * nst : 0;
        // two cells per pass keep more loads in flight (measured faster for
        // crweno5; hccs's heavier rows leave no room for it)
#pragma unroll(SCH == SCHEME_CR ? 2 : 1)
        for (int t = threadIdx.x; t < kCrTL * nst; t += kCrThreads) {
            int l, pc;
            if (DIR == 0) {
                if (t != (int)threadIdx.x) {
                    spc += kCrThreads;
                    while (spc >= nst) {
                        spc -= nst;
                        ++sl;
                    }
                }
                l = sl;
                pc = spc;
            } else {
                l = t % kCrTL;
                pc = t / kCrTL;
            }
            double fp = 0.0, fm = 0.0;
            if (l0 + l < nl) {
                int pos = pc - H;
                pos = pos < 0 ? pos + n : (pos >= n ? pos - n : pos);
                split(e, gidx(l, pos), fp, fm);
                if (mixed) {
                    fp = sub_(fp, sRef[0][e][l]);
                    fm = sub_(fm, sRef[1][e][l]);
                }
            }
            sF[l * ls + pc] = B(fp);
            sF[(kCrTL + l) * ls + pc] = B(fm);
        }
        __syncthreads();

        if (l0 + line < nl) {  // warp-uniform
            // explicit faces of the bounded system: 0..H-1 and n-H+1..n
            int xm = -1;
            B xv = B(0);
            // segment of this lane: rows r0 .. r1 (at least 2)
            const bool act = hl < P;
            const int r0 = act ? (hl * N) / P : 0;
            const int r1 = act ? ((hl + 1) * N) / P - 1 : 1;
            const int L = r1 - r0 + 1;
            B fa = B(0), fc = B(0), fd = B(0);  // reduced unit-diagonal row of x_first
            B la = B(0), lc = B(0), ld = B(0);  // reduced unit-diagonal row of x_last
            // the row work of one sign; the sign (warp-uniform) is a compile-time
            // constant inside, so each warp runs code without sign selects
            auto segment = [&](auto sign) {
                constexpr int S = decltype(sign)::value;
                auto F = [&](int c) -> B { return myF[c + H]; };
                // the sign (warp-uniform) only selects which cells feed a
                // stencil ('+' reads upwind from the left, '-' from the right)
                constexpr int dir = S == 0 ? 1 : -1;
                // explicit face m: WENO5-JS (crweno5.cpp:425-837), hccs's WENO7
                // (hccs.cpp:538-980) or hccs77's WENO7-Z (hccs77.cpp:330-818)
                auto js = [&](int m) -> B {
                    if (SCH == SCHEME_HC || SCH == SCHEME_H77) {
                        const int c0 = S == 0 ? m - 4 : m + 3;
                        if (SCH == SCHEME_HC)
                            return weno7_face_hc(F(c0), F(c0 + dir), F(c0 + 2 * dir),
                                                 F(c0 + 3 * dir), F(c0 + 4 * dir), F(c0 + 5 * dir),
                                                 F(c0 + 6 * dir));
                        return weno7_face(F(c0), F(c0 + dir), F(c0 + 2 * dir), F(c0 + 3 * dir),
                                          F(c0 + 4 * dir), F(c0 + 5 * dir), F(c0 + 6 * dir));
                    }
                    const int c0 = S == 0 ? m - 3 : m + 2;
                    return weno5js_face(F(c0), F(c0 + dir), F(c0 + 2 * dir), F(c0 + 3 * dir),
                                        F(c0 + 4 * dir));
                };
                // lanes 0..2H-1: the explicit faces; lanes 2H and 2H+1: the
                // identity rows' values (faces H and n-H), passed to the lanes
                // that own those rows, so the warp evaluates explicit faces once
                B did0 = B(0), did1 = B(0);
                if (bounded) {
                    B v = B(0);
                    if (hl < 2 * H + 2) {
                        const int m = hl < H ? hl
                                             : (hl < 2 * H ? n - 2 * H + 1 + hl
                                                           : (hl == 2 * H ? H : n - H));
                        v = js(m);
                        if (hl < 2 * H) {
                            xm = m;
                            xv = v;
                        }
                    }
                    did0 = shfl(v, 2 * H);
                    did1 = shfl(v, 2 * H + 1);
                }
                if (act) {
                    // window w[k] = F(i - WO + k) of the current row's cell i (face
                    // i + 1): cells i-2..i+3 for the 5-cell rows, i-3..i+4 for
                    // hccs77's 7-cell rows
                    constexpr int WN = SCH == SCHEME_H77 ? 8 : 6, WO = SCH == SCHEME_H77 ? 3 : 2;
                    int i = bounded ? r0 + H - 1 : r0 - 1;
                    B w[WN];
    #pragma unroll
                    for (int k = 0; k < WN; ++k) w[k] = F(i - WO + k);
                    // row r of the system; `ends`: r may be a bounded system's
                    // first or last row (identity rows)
                    auto gen = [&](int r, bool ends, B &a, B &b, B &c, B &d) {
                        if (ends && bounded && (r == 0 || r == N - 1)) {
                            a = B(0);
                            b = B(1);
                            c = B(0);
                            d = r == 0 ? did0 : did1;
                        } else {
                            // '+': cells i-2..i+2 = w[0..4]; '-': cells i+3..i-1 = w[5..1]
                            // with the off-diagonals swapped (crweno5.cpp:335-338)
                            constexpr bool m = S != 0;
                            B lo, hi;
                            if (SCH == SCHEME_H77)
                                // '+': cells i-3..i+3 = w[0..6]; '-': cells i+4..i-2 = w[7..1]
                                // (hccs77.cpp:282-291 swaps the couplings alike)
                                h77_row(w[m ? 7 : 0], w[m ? 6 : 1], w[m ? 5 : 2], w[m ? 4 : 3],
                                        w[m ? 3 : 4], w[m ? 2 : 5], w[m ? 1 : 6], lo, b, hi, d);
                            else if (SCH == SCHEME_HC)
                                hc_row(m ? w[5] : w[0], m ? w[4] : w[1], m ? w[3] : w[2],
                                       m ? w[2] : w[3], m ? w[1] : w[4], lo, b, hi, d);
                            else
                                cr_row(m ? w[5] : w[0], m ? w[4] : w[1], m ? w[3] : w[2],
                                       m ? w[2] : w[3], m ? w[1] : w[4], lo, b, hi, d);
                            a = m ? hi : lo;
                            c = m ? lo : hi;
                        }
                    };
                    auto advance = [&]() {
    #pragma unroll
                        for (int k = 0; k < WN - 1; ++k) w[k] = w[k + 1];
                        ++i;
                        w[WN - 1] = F(i + WN - 1 - WO);
                    };
                    B a0, b0, c0, d0;
                    gen(r0, true, a0, b0, c0, d0);
                    // forward: row j -> A x_first + x_j + C x_{j+1} = D.  Starting
                    // from (A, C, D) = (-1, 0, 0) makes row 1's update exact
                    // (b - a 0 = b, -a (-1) = a, d - a 0 = d), so every row takes
                    // the same code; only the last row can be an identity row.
                    B Ap = B(-1), Cp = B(0), Dp = B(0);
                    auto eliminate = [&](int j, B a, B b, B c, B d) {
                        const B bpv = b - a * Cp;
                        const B An = -a * Ap;
                        const B Dn = d - a * Dp;
                        const B r = rcp_(bpv);
                        Ap = An * r;
                        Cp = c * r;
                        Dp = Dn * r;
                        wA[j * 32 + lane] = Ap;
                        wC[j * 32 + lane] = Cp;
                        wD[j * 32 + lane] = Dp;
                    };
                    for (int j = 1; j < L - 1; ++j) {
                        advance();
                        B a, b, c, d;
                        gen(r0 + j, false, a, b, c, d);
                        eliminate(j, a, b, c, d);
                    }
                    {
                        advance();
                        B a, b, c, d;
                        gen(r0 + L - 1, true, a, b, c, d);
                        eliminate(L - 1, a, b, c, d);
                    }
                    la = Ap;
                    lc = Cp;
                    ld = Dp;
                    // backward: row j -> A x_first + x_j + C x_last = D
                    B bf = b0, cf = c0, df = d0;
                    if (L >= 3) {
                        B An = wA[(L - 2) * 32 + lane], Cn = wC[(L - 2) * 32 + lane];
                        B Dn = wD[(L - 2) * 32 + lane];
                        for (int j = L - 3; j >= 1; --j) {
                            const B k = wC[j * 32 + lane];
                            An = wA[j * 32 + lane] - k * An;
                            Cn = -k * Cn;
                            Dn = wD[j * 32 + lane] - k * Dn;
                            wA[j * 32 + lane] = An;
                            wC[j * 32 + lane] = Cn;
                            wD[j * 32 + lane] = Dn;
                        }
                        // row 0 minus c0 x (row 1)
                        bf = b0 - c0 * An;
                        cf = -c0 * Cn;
                        df = d0 - c0 * Dn;
                    }
                    const B r = rcp_(bf);
                    fa = a0 * r;
                    fc = cf * r;
                    fd = df * r;
                }
            };
            if (sg == 0)
                segment(std::integral_constant<int, 0>{});
            else
                segment(std::integral_constant<int, 1>{});
            // The 2P segment-end unknowns couple as
            //   fa x_last(l-1) + x_first(l) + fc x_last(l)  = fd   (lane l's first)
            //   la x_first(l)  + x_last(l)  + lc x_first(l+1) = ld (lane l's last)
            // (neighbour lanes wrap for periodic lines; for bounded lines lane
            // 0's fa and lane P-1's lc are 0: identity end rows).  Substituting
            // the first rows into the last rows leaves a tridiagonal system in
            // the P unknowns x_last alone,
            //   -la fa x_last(l-1) + (1 - la fc - lc fa') x_last(l) - lc fc' x_last(l+1)
            //     = ld - la fd - lc fd'          (' : lane l+1),
            // solved by parallel cyclic reduction with shuffles (log2 P levels
            // of one row each, instead of log2 2P levels of two rows); then
            // x_first(l) = fd - fa x_last(l-1) - fc x_last(l).
            B xf, xl;
            {
                // P is a power of two: lane indices wrap with a mask
                const int pm = P - 1;
                const int lp1 = (hl + 1) & pm, lm1 = (hl - 1) & pm;
                const B nfa = shfl(fa, lp1), nfc = shfl(fc, lp1), nfd = shfl(fd, lp1);
                const B r = rcp_(B(1) - la * fc - lc * nfa);
                B ra = -la * fa * r, rc = -lc * nfc * r, rd = (ld - la * fd - lc * nfd) * r;
#pragma unroll
                for (int s = 1; s < kCrLanes; s <<= 1) {
                    if (s >= P) break;  // warp-uniform
                    const int sm = (hl - s) & pm, sp = (hl + s) & pm;
                    B ma = shfl(ra, sm), mc = shfl(rc, sm), md = shfl(rd, sm);
                    B pa = shfl(ra, sp), pc = shfl(rc, sp), pd = shfl(rd, sp);
                    if (bounded && hl < s) ma = mc = md = B(0);
                    if (bounded && hl + s >= P) pa = pc = pd = B(0);
                    pcr_update(ra, rc, rd, ma, mc, md, pa, pc, pd);
                }
                // after the last level each row couples only to itself
                // (periodic) or to nothing (bounded)
                xl = rd * rcp_(B(1) + ra + rc);
                const B xlm = shfl(xl, lm1);
                xf = fd - fa * xlm - fc * xl;
            }
            __syncwarp();  // every lane has read its staged fluxes
            if (act) {
                const int off = bounded ? H : 0;
                myF[r0 + off] = xf;
                myF[r1 + off] = xl;
                for (int j = 1; j < L - 1; ++j)
                    myF[r0 + j + off] =
                        wD[j * 32 + lane] - wA[j * 32 + lane] * xf - wC[j * 32 + lane] * xl;
                if (!bounded && hl == 0) myF[n] = xf;  // face n is face 0
            }
            if (xm >= 0) myF[xm] = xv;
        }
        __syncthreads();
        // dF/dx of the tile's cells from F^ = F^+ + F^- (euler3d.cpp:23-56, 143-253)
        // four cells per thread and pass, their RHS loads issued together
        constexpr int U = 4;
        // x lines: (line, cell) of t = tid + m kCrThreads, advanced without a division
        int dl = DIR == 0 ? (int)threadIdx.x / n : 0;
        int di = DIR == 0 ? (int)threadIdx.x - dl * n : 0;
        for (int t0 = threadIdx.x; t0 < kCrTL * n; t0 += U * kCrThreads) {
            long long gi[U];
            B dfe[U], racc[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int t = t0 + u * kCrThreads;
                int l, i;
                if (DIR == 0) {
                    l = dl;
                    i = di;
                    di += kCrThreads;
                    while (di >= n) {
                        di -= n;
                        ++dl;
                    }
                } else {
                    l = t % kCrTL;
                    i = t / kCrTL;
                }
                gi[u] = -1;
                dfe[u] = racc[u] = B(0);
                if (t >= kCrTL * n || l0 + l >= nl) continue;
                const B *fp = sF + l * ls, *fm = sF + (kCrTL + l) * ls;
                dfe[u] = mul_(sub_(add_(fp[i + 1], fm[i + 1]), add_(fp[i], fm[i])), inv_d);
                gi[u] = (long long)e * np + gidx(l, i);
                if (accumulate) racc[u] = rbase[gi[u]];
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (gi[u] >= 0) rbase[gi[u]] = accumulate ? add_(racc[u], dfe[u]) : dfe[u];
        }
        __syncthreads();
    }
}

template <typename B, int SCH>
static cudaError_t prepare_t() {
    const int max_smem = 200 * 1024;  // above the largest need (166 KB at 512 cells, FP64)
    cudaError_t e = cudaFuncSetAttribute(k_crweno_lines<B, 0, SCH>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_crweno_lines<B, 1, SCH>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_crweno_lines<B, 2, SCH>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem);
    return e;
}

cudaError_t prepare_crweno_kernels(bool mixed) {
    cudaError_t e = mixed ? prepare_t<float, SCHEME_CR>() : prepare_t<double, SCHEME_CR>();
    if (e == cudaSuccess) e = mixed ? prepare_t<float, SCHEME_HC>() : prepare_t<double, SCHEME_HC>();
    if (e == cudaSuccess)
        e = mixed ? prepare_t<float, SCHEME_H77>() : prepare_t<double, SCHEME_H77>();
    return e;
}

template <typename B, int SCH>
static void launch_t(int dir, const BoxDev *boxes, const WorkItem *items, int nitems, int in_slot,
                     int accumulate, int nmax, int ms, int prim_mode, size_t smem,
                     cudaStream_t st) {
    if (dir == 0)
        k_crweno_lines<B, 0, SCH><<<nitems, kCrThreads, smem, st>>>(boxes, items, in_slot,
                                                                    accumulate, nmax, ms, prim_mode);
    else if (dir == 1)
        k_crweno_lines<B, 1, SCH><<<nitems, kCrThreads, smem, st>>>(boxes, items, in_slot,
                                                                    accumulate, nmax, ms, 0);
    else
        k_crweno_lines<B, 2, SCH><<<nitems, kCrThreads, smem, st>>>(boxes, items, in_slot,
                                                                    accumulate, nmax, ms, 0);
}

template <typename B>
cudaError_t launch_crweno(int sch, int dir, const BoxDev *boxes, const WorkItem *items,
                          int nitems, int in_slot, int accumulate, int nmax, int ms,
                          int prim_mode, cudaStream_t st) {
    if (nitems <= 0) return cudaSuccess;
    const size_t smem = crweno_smem_bytes(sch, nmax, ms, sizeof(B) == sizeof(float));
    if (sch == SCHEME_HC)
        launch_t<B, SCHEME_HC>(dir, boxes, items, nitems, in_slot, accumulate, nmax, ms, prim_mode,
                               smem, st);
    else if (sch == SCHEME_H77)
        launch_t<B, SCHEME_H77>(dir, boxes, items, nitems, in_slot, accumulate, nmax, ms,
                                prim_mode, smem, st);
    else
        launch_t<B, SCHEME_CR>(dir, boxes, items, nitems, in_slot, accumulate, nmax, ms, prim_mode,
                               smem, st);
    return cudaGetLastError();
}

template cudaError_t launch_crweno<double>(int, int, const BoxDev *, const WorkItem *, int, int,
                                           int, int, int, int, cudaStream_t);
template cudaError_t launch_crweno<float>(int, int, const BoxDev *, const WorkItem *, int, int,
                                          int, int, int, int, cudaStream_t);

}  // namespace nuc3d
