// Spectral shell forcing on the device, FP64: physicsModel::AddForcing_Const
// (physicsModel.cpp:1368-1641), called once per RHS evaluation after the RHS
// is assembled (NaiverStokes3d.cpp:58, euler3d.cpp:273).
//
// The reference transforms u, v, w with full 3-D FFTs (forward normalised by
// 1/N, backward unnormalised; fft.cpp:182-279), but only the modes of the
// shell |k - k_f| < 0.5 take part, so here the transforms are direct sums
// over the (2K+1)^3 wavevectors with |k_d| <= K = floor(k_f + 1/2), done as
// three separable passes each way against precomputed twiddle tables:
//   forward  x (one block per line) -> y -> z + mode algebra (one block)
//   backward z -> y -> x, the x pass fused with the RHS update.
// Per mode (physicsModel.cpp:1480-1531): the solenoidal part s = u^ - (k.u^)k
// / |k|^2 and the compressive part c = u^ - s; s gains the helical term
// sigma (i k x s) / |k|; the shell energies E_s, E_c (modes with
// |kmag' - k_f| < 0.5, kmag' = 1 at k = 0) give theta = sqrt(|A - E_c| / E_s)
// and the forcing spectrum s (theta - 1) on the modes with |kmag - k_f| < 0.5
// (kmag unmodified, so k = 0 counts in E_s but is not forced).  In physical
// space (rho taken as 1, physicsModel.cpp:1617-1640):
//   R[1..3] -= f,   R[4] -= f.u - <f.u>.
//
// The band forcing at a fixed injection rate (NUC3D_FORCING_BAND, not in the
// reference) shares every pass: on the modes with 0 < |k| <= k_f it forces
// the solenoidal part s (no helical term) as f = s P / (2 E_b), E_b the band's
// solenoidal energy sum |s|^2 / 2.  Since s is orthogonal to the compressive
// part, sum Re(f . conj(u^)) = P: the mean power <f.u> is P.
#include "forcing_kernels.h"

namespace nuc3d {

namespace {

constexpr int kThreads = 128;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// T[m * n + j] = exp(+i 2 pi k_m j / n), k_m = -K + m
__global__ void k_force_twiddle(double2 *T, int K, int n) {
    const int M = 2 * K + 1;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < M * n; t += gridDim.x * blockDim.x) {
        const int m = t / n, j = t % n;
        long long r = ((long long)(m - K) * j) % n;
        if (r < 0) r += n;
        double s, c;
        sincospi(2.0 * (double)r / (double)n, &s, &c);
        T[t] = make_double2(c, s);
    }
}

template <int NV>
__device__ void block_sum(double (&v)[NV], double *out) {
    __shared__ double red[NV][kThreads / 32];
    for (int i = 0; i < NV; ++i) {
        double s = v[i];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[i][threadIdx.x >> 5] = s;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NV; i += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) s += red[i][w];
        out[i] = s;
    }
    __syncthreads();
}

// forward x: A[c][m][line] = sum_i u_c(i, line) exp(-i 2 pi k_m i / nx)
template <int K>
__global__ void __launch_bounds__(kThreads) k_force_fx(BoxDev b, const double2 *Tx, double2 *A) {
    constexpr int M = 2 * K + 1;
    const BoxParams &p = b.p;
    const int nx = p.n[0];
    const long long lines = (long long)p.n[1] * p.n[2];
    const long long line = blockIdx.x;
    double acc[3 * M * 2];
#pragma unroll
    for (int s = 0; s < 3 * M * 2; ++s) acc[s] = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        const long long g = line * nx + i;
        const double u[3] = {fieldW(b, 0)[g], fieldW(b, 1)[g], fieldW(b, 2)[g]};
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const double2 t = Tx[m * nx + i];
#pragma unroll
            for (int c = 0; c < 3; ++c) {  // u * conj(t)
                acc[(c * M + m) * 2] += u[c] * t.x;
                acc[(c * M + m) * 2 + 1] -= u[c] * t.y;
            }
        }
    }
    __shared__ double out[3 * M * 2];
    block_sum<3 * M * 2>(acc, out);
    for (int s = threadIdx.x; s < 3 * M; s += blockDim.x)
        A[(long long)s * lines + line] = make_double2(out[2 * s], out[2 * s + 1]);
}

// forward y: B[c][mx][my][k] = sum_j A[c][mx][j + ny k] conj(Ty[my][j])
__global__ void k_force_fy(const double2 *A, const double2 *Ty, double2 *B, int K, int ny, int nz) {
    const int M = 2 * K + 1;
    const long long lines = (long long)ny * nz;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * M * M * nz; t += gridDim.x * blockDim.x) {
        const int k = t % nz, my = (t / nz) % M, cmx = t / (nz * M);  // cmx = c * M + mx
        double2 s = make_double2(0.0, 0.0);
        for (int j = 0; j < ny; ++j) {
            const double2 v = cmulc(A[(long long)cmx * lines + j + (long long)ny * k], Ty[my * ny + j]);
            s.x += v.x;
            s.y += v.y;
        }
        B[((long long)cmx * M + my) * nz + k] = s;
    }
}

__device__ __forceinline__ double kmag0_of(double kx, double ky, double kz) {
    return sqrt(kx * kx + ky * ky + kz * kz);
}

// forward z + mode algebra + shell energies + forcing spectrum (one block).
// scal: [0] E_s, [1] E_c, [2] theta, [3] <f.u> (set later)
__global__ void __launch_bounds__(kThreads)
    k_force_modes(const double2 *B, const double2 *Tz, double2 *Fh, double *scal, ForceParams fp,
                  int nx, int ny, int nz) {
    const int K = fp.K, M = 2 * K + 1, M3 = M * M * M;
    const double inv_n = 1.0 / ((double)nx * ny * nz);
    double e2[2] = {0.0, 0.0};
    // shared store of s (after the helical term) for the second loop
    extern __shared__ double2 sS[];  // [M3][3]
    for (int mode = threadIdx.x; mode < M3; mode += blockDim.x) {
        const int mx = mode % M, my = (mode / M) % M, mz = mode / (M * M);
        const double kx0 = mx - K, ky0 = my - K, kz0 = mz - K;
        double2 uh[3];
        for (int c = 0; c < 3; ++c) {
            double2 s = make_double2(0.0, 0.0);
            for (int k = 0; k < nz; ++k) {
                const double2 v = cmulc(B[(((long long)(c * M + mx)) * M + my) * nz + k], Tz[mz * nz + k]);
                s.x += v.x;
                s.y += v.y;
            }
            uh[c] = make_double2(s.x * inv_n, s.y * inv_n);  // fft.cpp:277-278
        }
        double kmag = sqrt(kx0 * kx0 + ky0 * ky0 + kz0 * kz0);
        if (kmag < 1e-6) kmag = 1.0;
        const double ku_re = (kx0 * uh[0].x + ky0 * uh[1].x + kz0 * uh[2].x) / kmag;
        const double ku_im = (kx0 * uh[0].y + ky0 * uh[1].y + kz0 * uh[2].y) / kmag;
        const double kk[3] = {kx0, ky0, kz0};
        double2 s[3], cc[3];
        for (int c = 0; c < 3; ++c) {
            s[c] = make_double2(uh[c].x - ku_re * kk[c] / kmag, uh[c].y - ku_im * kk[c] / kmag);
            cc[c] = make_double2(uh[c].x - s[c].x, uh[c].y - s[c].y);
        }
        if (fp.band) {
            // band forcing: the solenoidal part alone, energy over 0 < |k| <= k_f
            if (kmag0_of(kx0, ky0, kz0) > 0.0 && kmag0_of(kx0, ky0, kz0) <= fp.k + 1e-12)
                e2[0] += 0.5 * (s[0].x * s[0].x + s[1].x * s[1].x + s[2].x * s[2].x +
                                s[0].y * s[0].y + s[1].y * s[1].y + s[2].y * s[2].y);
            for (int c = 0; c < 3; ++c) sS[mode * 3 + c] = s[c];
            continue;
        }
        // helical term (physicsModel.cpp:1512-1526)
        const double kxu0_re = -(ky0 * s[2].y - kz0 * s[1].y) / kmag;
        const double kxu1_re = (kx0 * s[2].y - kz0 * s[0].y) / kmag;
        const double kxu2_re = -(kx0 * s[1].y - ky0 * s[0].y) / kmag;
        const double kxu0_im = (ky0 * s[2].x - kz0 * s[1].x) / kmag;
        const double kxu1_im = -(kx0 * s[2].x - kz0 * s[0].x) / kmag;
        const double kxu2_im = (kx0 * s[1].x - ky0 * s[0].x) / kmag;
        s[0] = make_double2(s[0].x + fp.hel * kxu0_re, s[0].y + fp.hel * kxu0_im);
        s[1] = make_double2(s[1].x + fp.hel * kxu1_re, s[1].y + fp.hel * kxu1_im);
        s[2] = make_double2(s[2].x + fp.hel * kxu2_re, s[2].y + fp.hel * kxu2_im);
        if (fabs(kmag - fp.k) < 0.5) {
            e2[0] += 0.5 * (s[0].x * s[0].x + s[1].x * s[1].x + s[2].x * s[2].x + s[0].y * s[0].y +
                            s[1].y * s[1].y + s[2].y * s[2].y);
            e2[1] += 0.5 * (cc[0].x * cc[0].x + cc[1].x * cc[1].x + cc[2].x * cc[2].x +
                            cc[0].y * cc[0].y + cc[1].y * cc[1].y + cc[2].y * cc[2].y);
        }
        for (int c = 0; c < 3; ++c) sS[mode * 3 + c] = s[c];
    }
    __shared__ double tot[2];
    block_sum<2>(e2, tot);
    // shell: theta - 1 multiplies the shell's modes; band: the gain P / (2 E_b)
    // (zero for a band without energy)
    const double theta = fp.band ? 0.0 : sqrt(fabs(fp.amp - tot[1]) / tot[0]);
    const double gain = fp.band ? (tot[0] > 0.0 ? fp.amp / (2.0 * tot[0]) : 0.0) : theta - 1.0;
    if (threadIdx.x == 0) {
        scal[0] = tot[0];
        scal[1] = tot[1];
        scal[2] = fp.band ? gain : theta;
    }
    for (int mode = threadIdx.x; mode < M3; mode += blockDim.x) {
        const int mx = mode % M, my = (mode / M) % M, mz = mode / (M * M);
        const double kx0 = mx - K, ky0 = my - K, kz0 = mz - K;
        const double kmag = kmag0_of(kx0, ky0, kz0);  // unmodified at k = 0
        const bool on = fp.band ? (kmag > 0.0 && kmag <= fp.k + 1e-12) : fabs(kmag - fp.k) < 0.5;
        for (int c = 0; c < 3; ++c) {
            const double2 s = sS[mode * 3 + c];
            Fh[c * M3 + mode] = on ? make_double2(s.x * gain, s.y * gain) : make_double2(0.0, 0.0);
        }
    }
}

// backward z: S[c][mx][my][k] = sum_mz Fh[c][mx,my,mz] Tz[mz][k]
__global__ void k_force_bz(const double2 *Fh, const double2 *Tz, double2 *S, int K, int nz) {
    const int M = 2 * K + 1, M3 = M * M * M;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * M * M * nz; t += gridDim.x * blockDim.x) {
        const int k = t % nz, my = (t / nz) % M, cmx = t / (nz * M);
        const int c = cmx / M, mx = cmx % M;
        double2 s = make_double2(0.0, 0.0);
        for (int mz = 0; mz < M; ++mz) {
            const double2 v = cmul(Fh[c * M3 + mx + M * (my + M * mz)], Tz[mz * nz + k]);
            s.x += v.x;
            s.y += v.y;
        }
        S[((long long)cmx * M + my) * nz + k] = s;
    }
}

// backward y: Y[c][mx][j + ny k] = sum_my S[c][mx][my][k] Ty[my][j]
__global__ void k_force_by(const double2 *S, const double2 *Ty, double2 *Y, int K, int ny, int nz) {
    const int M = 2 * K + 1;
    const long long lines = (long long)ny * nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3 * M * lines;
         t += (long long)gridDim.x * blockDim.x) {
        const long long line = t % lines;
        const int cmx = (int)(t / lines);
        const int j = (int)(line % ny), k = (int)(line / ny);
        double2 s = make_double2(0.0, 0.0);
        for (int my = 0; my < M; ++my) {
            const double2 v = cmul(S[((long long)cmx * M + my) * nz + k], Ty[my * ny + j]);
            s.x += v.x;
            s.y += v.y;
        }
        Y[t] = s;
    }
}

// backward x, per line: f_c(i) = Re sum_mx Y[c][mx][line] Tx[mx][i].  APPLY =
// false: per-line partial sums of f.u; true: the RHS update with <f.u>.
template <int K, bool APPLY, typename Bk>
__global__ void __launch_bounds__(kThreads)
    k_force_bx(BoxDev b, const double2 *Tx, const double2 *Y, double *partials, const double *scal) {
    constexpr int M = 2 * K + 1;
    const BoxParams &p = b.p;
    const int nx = p.n[0];
    const long long lines = (long long)p.n[1] * p.n[2];
    const long long line = blockIdx.x;
    __shared__ double2 sY[3 * M];
    for (int s = threadIdx.x; s < 3 * M; s += blockDim.x) sY[s] = Y[(long long)s * lines + line];
    __syncthreads();
    const double aver = APPLY ? scal[3] : 0.0;
    double acc[1] = {0.0};
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        double f[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < M; ++m) {
            const double2 t = Tx[m * nx + i];
#pragma unroll
            for (int c = 0; c < 3; ++c) f[c] += sY[c * M + m].x * t.x - sY[c * M + m].y * t.y;
        }
        const long long g = line * nx + i;
        const double u0 = fieldW(b, 0)[g], v0 = fieldW(b, 1)[g], w0 = fieldW(b, 2)[g];
        const double fu = f[0] * u0 + f[1] * v0 + f[2] * w0;  // rho0 = 1
        if (APPLY) {
            Bk *r = fieldR<Bk>(b, 0);
            const long long np = b.np;
            r[np + g] = Bk(double(r[np + g]) - f[0]);
            r[2 * np + g] = Bk(double(r[2 * np + g]) - f[1]);
            r[3 * np + g] = Bk(double(r[3 * np + g]) - f[2]);
            r[4 * np + g] = Bk(double(r[4 * np + g]) - (fu - aver));
        } else {
            acc[0] += fu;
        }
    }
    if (!APPLY) {
        __shared__ double out[1];
        block_sum<1>(acc, out);
        if (threadIdx.x == 0) partials[line] = out[0];
    }
}

// <f.u> = sum of the per-line partials / N (MPICommunicator.cpp:161-185), one block
__global__ void __launch_bounds__(kThreads) k_force_aver(const double *partials, long long lines,
                                                           double n_cells, double *scal) {
    double acc[1] = {0.0};
    for (long long l = threadIdx.x; l < lines; l += blockDim.x) acc[0] += partials[l];
    __shared__ double out[1];
    block_sum<1>(acc, out);
    if (threadIdx.x == 0) scal[3] = out[0] / n_cells;
}

int grid_for(long long n) {
    long long g = (n + 255) / 256;
    return (int)(g < 1 ? 1 : (g > 4096 ? 4096 : g));
}

template <int K, typename Bk>
cudaError_t launch_k(const BoxDev &b, const ForceScratch &s, ForceParams fp, cudaStream_t st) {
    const BoxParams &p = b.p;
    const int nx = p.n[0], ny = p.n[1], nz = p.n[2];
    const long long lines = (long long)ny * nz;
    constexpr int M = 2 * K + 1;
    k_force_fx<K><<<(unsigned)lines, kThreads, 0, st>>>(b, s.tx, s.a);
    k_force_fy<<<grid_for(3LL * M * M * nz), 256, 0, st>>>(s.a, s.ty, s.b, K, ny, nz);
    k_force_modes<<<1, kThreads, sizeof(double2) * 3 * M * M * M, st>>>(s.b, s.tz, s.fh, s.scal, fp,
                                                                         nx, ny, nz);
    k_force_bz<<<grid_for(3LL * M * M * nz), 256, 0, st>>>(s.fh, s.tz, s.b, K, nz);
    k_force_by<<<grid_for(3LL * M * lines), 256, 0, st>>>(s.b, s.ty, s.a, K, ny, nz);
    k_force_bx<K, false, Bk><<<(unsigned)lines, kThreads, 0, st>>>(b, s.tx, s.a, s.partials, s.scal);
    k_force_aver<<<1, kThreads, 0, st>>>(s.partials, lines, (double)p.N, s.scal);
    k_force_bx<K, true, Bk><<<(unsigned)lines, kThreads, 0, st>>>(b, s.tx, s.a, s.partials, s.scal);
    return cudaGetLastError();
}

}  // namespace

int forcing_K(double k_f) { return (int)std::floor(k_f + 0.5); }

size_t forcing_scratch_bytes(const BoxParams &p, double k_f) {
    const int K = forcing_K(k_f), M = 2 * K + 1;
    const long long lines = (long long)p.n[1] * p.n[2];
    size_t b = 0;
    b += sizeof(double2) * (size_t)M * (p.n[0] + p.n[1] + p.n[2]);  // twiddles
    b += sizeof(double2) * 3 * (size_t)M * lines;                   // a
    b += sizeof(double2) * 3 * (size_t)M * M * p.n[2];              // b
    b += sizeof(double2) * 3 * (size_t)M * M * M;                   // fh
    b += sizeof(double) * (size_t)lines + 8 * sizeof(double);       // partials, scal
    return b + 8 * 256;
}

ForceScratch forcing_layout(const BoxParams &p, double k_f, void *base) {
    const int K = forcing_K(k_f), M = 2 * K + 1;
    const long long lines = (long long)p.n[1] * p.n[2];
    char *c = static_cast<char *>(base);
    auto take = [&](size_t bytes) {
        char *r = c;
        c += (bytes + 255) / 256 * 256;
        return r;
    };
    ForceScratch s{};
    s.tx = reinterpret_cast<double2 *>(take(sizeof(double2) * M * p.n[0]));
    s.ty = reinterpret_cast<double2 *>(take(sizeof(double2) * M * p.n[1]));
    s.tz = reinterpret_cast<double2 *>(take(sizeof(double2) * M * p.n[2]));
    s.a = reinterpret_cast<double2 *>(take(sizeof(double2) * 3 * (size_t)M * lines));
    s.b = reinterpret_cast<double2 *>(take(sizeof(double2) * 3 * (size_t)M * M * p.n[2]));
    s.fh = reinterpret_cast<double2 *>(take(sizeof(double2) * 3 * (size_t)M * M * M));
    s.partials = reinterpret_cast<double *>(take(sizeof(double) * (size_t)lines));
    s.scal = reinterpret_cast<double *>(take(8 * sizeof(double)));
    return s;
}

cudaError_t forcing_prepare(const BoxParams &p, double k_f, const ForceScratch &s, cudaStream_t st) {
    const int K = forcing_K(k_f), M = 2 * K + 1;
    k_force_twiddle<<<grid_for((long long)M * p.n[0]), 256, 0, st>>>(s.tx, K, p.n[0]);
    k_force_twiddle<<<grid_for((long long)M * p.n[1]), 256, 0, st>>>(s.ty, K, p.n[1]);
    k_force_twiddle<<<grid_for((long long)M * p.n[2]), 256, 0, st>>>(s.tz, K, p.n[2]);
    return cudaGetLastError();
}

template <typename Bk>
cudaError_t launch_forcing(const BoxDev &b, const ForceScratch &s, ForceParams fp, cudaStream_t st) {
    switch (fp.K) {
        case 0: return launch_k<0, Bk>(b, s, fp, st);
        case 1: return launch_k<1, Bk>(b, s, fp, st);
        case 2: return launch_k<2, Bk>(b, s, fp, st);
        case 3: return launch_k<3, Bk>(b, s, fp, st);
        default: return cudaErrorInvalidValue;
    }
}

template cudaError_t launch_forcing<double>(const BoxDev &, const ForceScratch &, ForceParams,
                                            cudaStream_t);
template cudaError_t launch_forcing<float>(const BoxDev &, const ForceScratch &, ForceParams,
                                           cudaStream_t);

}  // namespace nuc3d
