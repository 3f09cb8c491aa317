// Initial states generated on the device, so a solve can start without a
// host-side field or a host->device copy of one.
//
//   Taylor-Green vortex   block::initial_taylorgreen (block.cpp:359-395)
//   decaying isotropic    block::initial_hit (block.cpp:397-551)
//   turbulence (HIT)
//
// HIT: the reference fills every FFT index with a random-phase solenoidal
// coefficient (Craya-Herring projection, E(k) ~ (k/kp)^4 exp(-2 (k/kp)^2),
// three phases per mode from std::mt19937 in index order), transforms back
// with an unnormalised complex FFT and keeps the real part, then rescales to
// the target rms velocity.  Here the phases come from a counter-based stream
// (splitmix64 output 3*idx + c + 1, idx the FFT index of the mode), so they
// can be drawn in parallel, and the backward transform is a direct synthesis
// restricted to |k_d| <= 6.5 kp on each axis: a mode outside has amplitude
// below 1e-17 of the peak, so the truncation is below FP64 rounding.  The
// synthesis runs as three separable passes (z, y, x), each a short complex
// dot product per output point against a precomputed twiddle table, with the
// Taylor-microscale derivatives (postproc.cpp:871) formed on the way.
#include <cuda_runtime.h>

#include "init_kernels.h"

namespace nuc3d {

namespace {

constexpr double kPi = 3.141592653589793;  // 4 atan(1) (block.cpp:413)

__device__ __forceinline__ double unit_splitmix(unsigned long long seed, unsigned long long n) {
    unsigned long long z = seed + n * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
    return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}

// i * f * c
__device__ __forceinline__ double2 imul(double f, double2 c) {
    return make_double2(-__dmul_rn(f, c.y), __dmul_rn(f, c.x));
}

// ---------------------------------------------------------------- TGV ----
__global__ void k_init_tgv(BoxDev b) {
    const BoxParams &p = b.p;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < p.N;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % p.n[0]);
        const int j = (int)((c / p.n[0]) % p.n[1]);
        const int k = (int)(c / ((long long)p.n[0] * p.n[1]));
        // cell centres x = dx (i + 1/2) - x0 with x0 = 0 (block.cpp:103-124)
        const double x = __dmul_rn(p.d[0], 0.5 + i);
        const double y = __dmul_rn(p.d[1], 0.5 + j);
        const double z = __dmul_rn(p.d[2], 0.5 + k);
        const double g = p.gamma, M = p.mach;
        const double u0 = __dmul_rn(__dmul_rn(sin(x), cos(y)), cos(z));
        const double v0 = __dmul_rn(__dmul_rn(-cos(x), sin(y)), cos(z));
        const double w0 = 0.0;
        const double p0 = __dadd_rn(
            1.0 / __dmul_rn(__dmul_rn(g, M), M),
            __dsub_rn(__dmul_rn(__dadd_rn(cos(2.0 * z), 2.0), __dadd_rn(cos(2.0 * x), cos(2.0 * y))),
                      2.0) / 16.0);
        const double ke = __dadd_rn(__dadd_rn(__dmul_rn(u0, u0), __dmul_rn(v0, v0)), __dmul_rn(w0, w0));
        fieldU(b, 0, 0)[c] = 1.0;
        fieldU(b, 0, 1)[c] = u0;
        fieldU(b, 0, 2)[c] = v0;
        fieldU(b, 0, 3)[c] = w0;
        fieldU(b, 0, 4)[c] = __dadd_rn(p0 / (g - 1.0), __dmul_rn(0.5, ke));
    }
}

// ---------------------------------------------------------------- HIT ----
// T[m * n + j] = exp(+i 2 pi k_m j / n), k_m = kmin + m; the phase is
// reduced exactly ((k j) mod n) before the sine/cosine.
__global__ void k_hit_twiddle(double2 *T, HitAxis ax) {
    const long long total = (long long)ax.M * ax.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(t / ax.n), j = (int)(t % ax.n);
        long long r = ((long long)(ax.kmin + m) * j) % ax.n;
        if (r < 0) r += ax.n;
        double s, c;
        sincospi(2.0 * (double)r / (double)ax.n, &s, &c);
        T[t] = make_double2(c, s);
    }
}

// Spectral coefficients of u, v, w for the retained modes (block.cpp:466-497).
__global__ void k_hit_coeff(double2 *C, HitAxis ax, HitAxis ay, HitAxis az,
                            unsigned long long seed, double k_peak, double u_rms) {
    const long long Mxy = (long long)ax.M * ay.M, total = Mxy * az.M;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int mx = (int)(t % ax.M), my = (int)((t / ax.M) % ay.M), mz = (int)(t / Mxy);
        const int ikx = ax.kmin + mx, iky = ay.kmin + my, ikz = az.kmin + mz;
        const double kx0 = ikx, ky0 = iky, kz0 = ikz;
        const unsigned long long ix = ikx < 0 ? ikx + ax.n : ikx;
        const unsigned long long iy = iky < 0 ? iky + ay.n : iky;
        const unsigned long long iz = ikz < 0 ? ikz + az.n : ikz;
        const unsigned long long idx = ix + (unsigned long long)ax.n * (iy + (unsigned long long)ay.n * iz);
        double kmag = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(kx0, kx0), __dmul_rn(ky0, ky0)), __dmul_rn(kz0, kz0)));
        const double k12 = sqrt(__dadd_rn(__dmul_rn(kx0, kx0), __dmul_rn(ky0, ky0)));
        if (kmag < 1e-6) kmag = 1.0;
        const double q = kmag / k_peak;
        const double ek = __dmul_rn(__dmul_rn(u_rms * u_rms * 16.0 * sqrt(2.0 / kPi), pow(q, 4.0)) / k_peak,
                                    exp(-2.0 * kmag * kmag / k_peak / k_peak));
        const double amp = sqrt(2.0 * ek / kmag / kmag / 4.0 / kPi);
        const double phi1 = 2.0 * kPi * unit_splitmix(seed, 3 * idx + 1);
        const double phi2 = 2.0 * kPi * unit_splitmix(seed, 3 * idx + 2);
        const double phi3 = 2.0 * kPi * unit_splitmix(seed, 3 * idx + 3);
        const double c3 = cos(phi3), s3 = sin(phi3);
        const double2 a = make_double2(__dmul_rn(__dmul_rn(amp, cos(phi1)), c3),
                                       __dmul_rn(__dmul_rn(amp, sin(phi1)), c3));
        const double2 bb = make_double2(__dmul_rn(__dmul_rn(amp, cos(phi2)), s3),
                                        __dmul_rn(__dmul_rn(amp, sin(phi2)), s3));
        const bool axis = k12 < 1e-6;
        const double k212 = axis ? 1.0 : ky0 / k12;
        const double k112 = axis ? 0.0 : kx0 / k12;
        const double fu = __dmul_rn(k112, kz0) / kmag;  // multiplies b in u
        const double fv = __dmul_rn(k212, kz0) / kmag;  // multiplies b in v
        const double fw = -k12 / kmag;
        C[t] = make_double2(__dadd_rn(__dmul_rn(k212, a.x), __dmul_rn(fu, bb.x)),
                            __dadd_rn(__dmul_rn(k212, a.y), __dmul_rn(fu, bb.y)));
        C[total + t] = make_double2(__dsub_rn(__dmul_rn(fv, bb.x), __dmul_rn(k112, a.x)),
                                    __dsub_rn(__dmul_rn(fv, bb.y), __dmul_rn(k112, a.y)));
        C[2 * total + t] = make_double2(__dmul_rn(fw, bb.x), __dmul_rn(fw, bb.y));
    }
}

// Derivative factor of wavenumber k on an axis of n points and length L:
// 2 pi k / L, and 0 at the Nyquist wavenumber (a spectral derivative of the
// real field has no Nyquist part).
__device__ __forceinline__ double dfac(int k, const HitAxis &a) {
    return 2 * (k < 0 ? -k : k) == a.n ? 0.0 : (double)k * a.kscale;
}

// Pass z: A[f][z][my][mx] = sum_mz C[f][mz][my][mx] T_z[mz][z], f = u, v, w,
// dw/dz.
__global__ void k_hit_synth_z(const double2 *__restrict__ C, const double2 *__restrict__ Tz,
                              double2 *__restrict__ A, HitAxis ax, HitAxis ay, HitAxis az) {
    const long long Mxy = (long long)ax.M * ay.M, cstride = Mxy * az.M, astride = Mxy * az.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < astride;
         t += (long long)gridDim.x * blockDim.x) {
        const long long mxy = t % Mxy;
        const int z = (int)(t / Mxy);
        double2 su = {0, 0}, sv = {0, 0}, sw = {0, 0}, swz = {0, 0};
        for (int mz = 0; mz < az.M; ++mz) {
            const double2 tw = Tz[(long long)mz * az.n + z];
            const long long ci = mz * Mxy + mxy;
            const double2 cw = cmul(C[2 * cstride + ci], tw);
            su = cadd(su, cmul(C[ci], tw));
            sv = cadd(sv, cmul(C[cstride + ci], tw));
            sw = cadd(sw, cw);
            swz = cadd(swz, imul(dfac(az.kmin + mz, az), cw));
        }
        A[t] = su;
        A[astride + t] = sv;
        A[2 * astride + t] = sw;
        A[3 * astride + t] = swz;
    }
}

// Pass y: B[g][z][y][mx] = sum_my A[.][z][my][mx] T_y[my][y], g = u, v, w,
// dv/dy, dw/dz.
__global__ void k_hit_synth_y(const double2 *__restrict__ A, const double2 *__restrict__ Ty,
                              double2 *__restrict__ Bf, HitAxis ax, HitAxis ay, HitAxis az) {
    const long long astride = (long long)ax.M * ay.M * az.n;
    const long long bstride = (long long)ax.M * ay.n * az.n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < bstride;
         t += (long long)gridDim.x * blockDim.x) {
        const int mx = (int)(t % ax.M);
        const int y = (int)((t / ax.M) % ay.n);
        const int z = (int)(t / ((long long)ax.M * ay.n));
        double2 su = {0, 0}, sv = {0, 0}, sw = {0, 0}, svy = {0, 0}, swz = {0, 0};
        const long long a0 = (long long)z * ay.M * ax.M + mx;
        for (int my = 0; my < ay.M; ++my) {
            const double2 tw = Ty[(long long)my * ay.n + y];
            const long long ai = a0 + (long long)my * ax.M;
            const double2 cv = cmul(A[astride + ai], tw);
            su = cadd(su, cmul(A[ai], tw));
            sv = cadd(sv, cv);
            sw = cadd(sw, cmul(A[2 * astride + ai], tw));
            svy = cadd(svy, imul(dfac(ay.kmin + my, ay), cv));
            swz = cadd(swz, cmul(A[3 * astride + ai], tw));
        }
        Bf[t] = su;
        Bf[bstride + t] = sv;
        Bf[2 * bstride + t] = sw;
        Bf[3 * bstride + t] = svy;
        Bf[4 * bstride + t] = swz;
    }
}

constexpr int kSynthThreads = 128;

// Fixed-order block sum of NV values per thread (deterministic).
template <int NV>
__device__ void block_sum(double (&v)[NV], double *out) {
    __shared__ double red[NV][kSynthThreads / 32];
    for (int i = 0; i < NV; ++i) {
        double s = v[i];
        for (int o = 16; o > 0; o >>= 1) s = __dadd_rn(s, __shfl_down_sync(0xffffffffu, s, o));
        if ((threadIdx.x & 31) == 0) red[i][threadIdx.x >> 5] = s;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int w = 0; w < kSynthThreads / 32; ++w) s = __dadd_rn(s, red[threadIdx.x][w]);
        out[threadIdx.x] = s;
    }
}

// Pass x: one block per (y, z) line.  Writes the raw (unscaled) velocity
// and the line's sums of u^2, v^2, w^2, u_x^2, v_y^2, w_z^2.
__global__ void __launch_bounds__(kSynthThreads)
    k_hit_synth_x(const double2 *__restrict__ Bf, const double2 *__restrict__ Tx, double *u,
                  double *v, double *w, double *partials, HitAxis ax, HitAxis ay, HitAxis az) {
    extern __shared__ double2 sB[];  // [5][Mx]
    const long long line = blockIdx.x;  // y + ny z
    const long long bstride = (long long)ax.M * ay.n * az.n;
    for (int i = threadIdx.x; i < 5 * ax.M; i += blockDim.x) {
        const int g = i / ax.M, m = i % ax.M;
        sB[i] = Bf[g * bstride + line * ax.M + m];
    }
    __syncthreads();
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int x = threadIdx.x; x < ax.n; x += blockDim.x) {
        double fu = 0, fv = 0, fw = 0, fux = 0, fvy = 0, fwz = 0;
        for (int m = 0; m < ax.M; ++m) {
            const double2 tw = Tx[(long long)m * ax.n + x];
            const double2 pu = cmul(sB[m], tw);
            fu = __dadd_rn(fu, pu.x);
            fv = __dadd_rn(fv, cmul(sB[ax.M + m], tw).x);
            fw = __dadd_rn(fw, cmul(sB[2 * ax.M + m], tw).x);
            fux = __dadd_rn(fux, imul(dfac(ax.kmin + m, ax), pu).x);
            fvy = __dadd_rn(fvy, cmul(sB[3 * ax.M + m], tw).x);
            fwz = __dadd_rn(fwz, cmul(sB[4 * ax.M + m], tw).x);
        }
        const long long c = line * ax.n + x;
        u[c] = fu;
        v[c] = fv;
        w[c] = fw;
        acc[0] = __dadd_rn(acc[0], __dmul_rn(fu, fu));
        acc[1] = __dadd_rn(acc[1], __dmul_rn(fv, fv));
        acc[2] = __dadd_rn(acc[2], __dmul_rn(fw, fw));
        acc[3] = __dadd_rn(acc[3], __dmul_rn(fux, fux));
        acc[4] = __dadd_rn(acc[4], __dmul_rn(fvy, fvy));
        acc[5] = __dadd_rn(acc[5], __dmul_rn(fwz, fwz));
    }
    block_sum<6>(acc, partials + line * 6);
}

// Sum of the per-line partials, one block, fixed order.
__global__ void __launch_bounds__(kSynthThreads) k_hit_reduce(const double *partials, long long nlines,
                                                               double *out) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (long long l = threadIdx.x; l < nlines; l += blockDim.x)
        for (int i = 0; i < 6; ++i) acc[i] = __dadd_rn(acc[i], partials[l * 6 + i]);
    block_sum<6>(acc, out);
}

// Conserved state from the scaled velocity (block.cpp:531-546).
__global__ void k_hit_finalize(BoxDev b, const double *u, const double *v, const double *w,
                               double scale) {
    const BoxParams &p = b.p;
    const double g = p.gamma, M = p.mach;
    const double p0 = 1.0 / __dmul_rn(__dmul_rn(g, M), M);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < p.N;
         c += (long long)gridDim.x * blockDim.x) {
        const double u0 = __dmul_rn(u[c], scale), v0 = __dmul_rn(v[c], scale), w0 = __dmul_rn(w[c], scale);
        const double ke = __dadd_rn(__dadd_rn(__dmul_rn(u0, u0), __dmul_rn(v0, v0)), __dmul_rn(w0, w0));
        fieldU(b, 0, 0)[c] = 1.0;
        fieldU(b, 0, 1)[c] = u0;
        fieldU(b, 0, 2)[c] = v0;
        fieldU(b, 0, 3)[c] = w0;
        fieldU(b, 0, 4)[c] = __dadd_rn(p0 / (g - 1.0), __dmul_rn(0.5, ke));
    }
}

int grid_for(long long n) {
    long long g = (n + 255) / 256;
    return (int)(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

}  // namespace

HitAxis hit_axis(int n, double length, double k_peak) {
    HitAxis a{};
    a.n = n;
    a.kscale = 2.0 * kPi / length;
    int kc = (int)(6.5 * k_peak + 1.0);
    if (kc > n / 2) kc = n / 2;
    a.kmin = -kc;
    const int kmax = (2 * kc == n) ? kc - 1 : kc;  // index n/2 is wavenumber -n/2
    a.M = kmax - a.kmin + 1;
    return a;
}

size_t hit_scratch_bytes(const BoxParams &p, double k_peak) {
    HitAxis ax = hit_axis(p.n[0], 1.0, k_peak), ay = hit_axis(p.n[1], 1.0, k_peak),
            az = hit_axis(p.n[2], 1.0, k_peak);
    size_t c2 = sizeof(double2);
    size_t b = 3 * (size_t)ax.M * ay.M * az.M * c2;
    b += 4 * (size_t)ax.M * ay.M * p.n[2] * c2;
    b += 5 * (size_t)ax.M * p.n[1] * p.n[2] * c2;
    b += ((size_t)ax.M * ax.n + (size_t)ay.M * ay.n + (size_t)az.M * az.n) * c2;
    b += (size_t)p.n[1] * p.n[2] * 6 * sizeof(double) + 8 * sizeof(double);
    return b + 8 * 256;
}

cudaError_t launch_init_tgv(const BoxDev &b, cudaStream_t st) {
    k_init_tgv<<<grid_for(b.p.N), 256, 0, st>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_hit_synthesis(const BoxDev &b, double lx, double ly, double lz,
                                 unsigned long long seed, double k_peak, double u_rms,
                                 void *scratch, double *d_sums, cudaStream_t st) {
    const BoxParams &p = b.p;
    HitAxis ax = hit_axis(p.n[0], lx, k_peak), ay = hit_axis(p.n[1], ly, k_peak),
            az = hit_axis(p.n[2], lz, k_peak);
    char *s = static_cast<char *>(scratch);
    auto take = [&](size_t bytes) {
        char *r = s;
        s += (bytes + 255) / 256 * 256;
        return r;
    };
    const long long nC = (long long)ax.M * ay.M * az.M;
    const long long nA = (long long)ax.M * ay.M * p.n[2];
    const long long nB = (long long)ax.M * p.n[1] * p.n[2];
    double2 *C = reinterpret_cast<double2 *>(take(3 * nC * sizeof(double2)));
    double2 *A = reinterpret_cast<double2 *>(take(4 * nA * sizeof(double2)));
    double2 *Bf = reinterpret_cast<double2 *>(take(5 * nB * sizeof(double2)));
    double2 *Tx = reinterpret_cast<double2 *>(take((size_t)ax.M * ax.n * sizeof(double2)));
    double2 *Ty = reinterpret_cast<double2 *>(take((size_t)ay.M * ay.n * sizeof(double2)));
    double2 *Tz = reinterpret_cast<double2 *>(take((size_t)az.M * az.n * sizeof(double2)));
    const long long nlines = (long long)p.n[1] * p.n[2];
    double *partials = reinterpret_cast<double *>(take(nlines * 6 * sizeof(double)));
    k_hit_twiddle<<<grid_for((long long)ax.M * ax.n), 256, 0, st>>>(Tx, ax);
    k_hit_twiddle<<<grid_for((long long)ay.M * ay.n), 256, 0, st>>>(Ty, ay);
    k_hit_twiddle<<<grid_for((long long)az.M * az.n), 256, 0, st>>>(Tz, az);
    k_hit_coeff<<<grid_for(nC), 256, 0, st>>>(C, ax, ay, az, seed, k_peak, u_rms);
    k_hit_synth_z<<<grid_for(nA), 256, 0, st>>>(C, Tz, A, ax, ay, az);
    k_hit_synth_y<<<grid_for(nB), 256, 0, st>>>(A, Ty, Bf, ax, ay, az);
    k_hit_synth_x<<<(unsigned)nlines, kSynthThreads, 5 * ax.M * sizeof(double2), st>>>(
        Bf, Tx, fieldW(b, 0), fieldW(b, 1), fieldW(b, 2), partials, ax, ay, az);
    k_hit_reduce<<<1, kSynthThreads, 0, st>>>(partials, nlines, d_sums);
    return cudaGetLastError();
}

cudaError_t launch_hit_finalize(const BoxDev &b, double scale, cudaStream_t st) {
    k_hit_finalize<<<grid_for(b.p.N), 256, 0, st>>>(b, fieldW(b, 0), fieldW(b, 1), fieldW(b, 2), scale);
    return cudaGetLastError();
}

}  // namespace nuc3d
