// Shell-binned spectra of a box's current state: postproc::solveFFT
// (postproc.cpp:931-1184) with fft::solveFFT_forward (fft.cpp:182-283) and the
// two fft::solveShell binnings (fft.cpp:384-572), FP64.
//
//   k_spec_fields  u, v, w, the helicity field w.u, the enstrophy field
//                  |w|^2/2 (solveQ's fields, postproc.cpp:812-853, vorticity
//                  from the differential scheme's gradients), density and pressure, as complex
//                  fields with zero imaginary part;
//   cuFFT          one batched forward 3-D Z2Z transform of the seven fields
//                  (FFTW_FORWARD sign; the 1/N of fft.cpp:277-278 is applied
//                  when binning);
//   k_spec_bin     per mode: the folded wavenumber, the compressive /
//                  solenoidal / helical split of the velocity transform
//                  (postproc.cpp:1013-1101) and the shell of each binning.
//                  The kinetic spectra use the folded |k| with |k| = 1
//                  substituted at k = 0 (fft.cpp:424-435, the mean flow lands
//                  in shell 1); the scalar spectra use the unfolded
//                  i^2 + j^2 + k^2 of fft.cpp:517-531 (only the non-negative
//                  octant is counted).  Each block adds its modes into shared
//                  shell sums in a fixed order;
//   k_spec_reduce  adds the blocks' shell sums in a fixed order.
// The grid is fixed, so a box gives the same bits alone or in any batch.
#include <cufft.h>

#include "nuc3d_device.cuh"
#include "spectra_kernels.h"

namespace nuc3d {

namespace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_spec_fields(BoxDev b, double2 *F) {
    const BoxParams &p = b.p;
    const long long N = p.N;
    const double *rho = fieldU(b, 0, 0);
    const double *u = fieldW(b, 0), *v = fieldW(b, 1), *w = fieldW(b, 2), *pr = fieldW(b, 3);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % p.n[0]);
        const int j = (int)((c / p.n[0]) % p.n[1]);
        const int k = (int)(c / ((long long)p.n[0] * p.n[1]));
        const double u0 = u[c], u1 = v[c], u2 = w[c];
        const double uy = diff_at(u, p, i, j, k, 1), uz = diff_at(u, p, i, j, k, 2);
        const double vx = diff_at(v, p, i, j, k, 0), vz = diff_at(v, p, i, j, k, 2);
        const double wx = diff_at(w, p, i, j, k, 0), wy = diff_at(w, p, i, j, k, 1);
        const double w0 = wy - vz, w1 = uz - wx, w2 = vx - uy;
        F[c] = make_double2(u0, 0.0);
        F[N + c] = make_double2(u1, 0.0);
        F[2 * N + c] = make_double2(u2, 0.0);
        F[3 * N + c] = make_double2(w0 * u0 + w1 * u1 + w2 * u2, 0.0);
        F[4 * N + c] = make_double2((w0 * w0 + w1 * w1 + w2 * w2) * 0.5, 0.0);
        F[5 * N + c] = make_double2(rho[c], 0.0);
        F[6 * N + c] = make_double2(pr[c], 0.0);
    }
}

// shell of |k| (fft.cpp:432-433): floor(|k|), or floor + 1 past the half
__device__ __forceinline__ int shell_of(double kmag) {
    const double fl = floor(kmag);
    return ((kmag - fl) - 0.5 <= 0) ? (int)fl : (int)fl + 1;
}

__device__ __forceinline__ double folded(int i, int n) {
    return (i >= n / 2.0) ? (double)i - n : (double)i;  // fft.cpp:424-426
}

__device__ __forceinline__ double sq(double x) { return x * x; }

__global__ void __launch_bounds__(kThreads) k_spec_bin(const double2 *F, int nx, int ny, int nz,
                                                        int kmax, double *partials) {
    extern __shared__ __align__(16) double sm[];
    const int ks = kmax + 1;
    double *hist = sm;                        // [kSpectra][kmax + 1]
    double *val = hist + kSpectra * ks;       // [kSpectra][kThreads]
    int *shell = reinterpret_cast<int *>(val + kSpectra * kThreads);  // [2][kThreads]
    for (int t = threadIdx.x; t < kSpectra * ks; t += blockDim.x) hist[t] = 0.0;
    const long long N = (long long)nx * ny * nz;
    const long long chunk = (N + gridDim.x - 1) / gridDim.x;
    const long long m0 = blockIdx.x * chunk;
    const long long m1 = m0 + chunk < N ? m0 + chunk : N;
    const double dN = (double)N;
    __syncthreads();
    for (long long base = m0; base < m1; base += kThreads) {
        const long long m = base + threadIdx.x;
        int sk = -1, so = -1;
        double v[kSpectra];
#pragma unroll
        for (int q = 0; q < kSpectra; ++q) v[q] = 0.0;
        if (m < m1) {
            const int i = (int)(m % nx), j = (int)((m / nx) % ny), k = (int)(m / ((long long)nx * ny));
            const double kx = folded(i, nx), ky = folded(j, ny), kz = folded(k, nz);
            double kmag = sqrt(kx * kx + ky * ky + kz * kz);
            if (kmag < 1e-6) kmag = 1.0;
            if (kmag < kmax) {
                sk = shell_of(kmag);
                double ur[3], ui[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double2 f = F[d * N + m];
                    ur[d] = f.x / dN;  // fft.cpp:277-278 (division, as normalization())
                    ui[d] = f.y / dN;
                }
                const double kv[3] = {kx, ky, kz};
                const double ku_r = (kx * ur[0] + ky * ur[1] + kz * ur[2]) / kmag;
                const double ku_i = (kx * ui[0] + ky * ui[1] + kz * ui[2]) / kmag;
                double sr[3], si[3], cr[3], ci[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    sr[d] = ur[d] - ku_r * kv[d] / kmag;
                    si[d] = ui[d] - ku_i * kv[d] / kmag;
                    cr[d] = ur[d] - sr[d];
                    ci[d] = ui[d] - si[d];
                }
                // i k x s / |k| (postproc.cpp:1052-1059)
                const double xr[3] = {-(ky * si[2] - kz * si[1]) / kmag,
                                      (kx * si[2] - kz * si[0]) / kmag,
                                      -(kx * si[1] - ky * si[0]) / kmag};
                const double xi[3] = {(ky * sr[2] - kz * sr[1]) / kmag,
                                      -(kx * sr[2] - kz * sr[0]) / kmag,
                                      (kx * sr[1] - ky * sr[0]) / kmag};
                double e[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    e[0] += sq(ur[d]) + sq(ui[d]);
                    e[1] += sq(cr[d]) + sq(ci[d]);
                    e[2] += sq(sr[d]) + sq(si[d]);
                    e[3] += sq(0.5 * (sr[d] - xr[d])) + sq(0.5 * (si[d] - xi[d]));
                    e[4] += sq(0.5 * (sr[d] + xr[d])) + sq(0.5 * (si[d] + xi[d]));
                }
#pragma unroll
                for (int q = 0; q < 5; ++q) v[q] = 0.5 * e[q];
            }
            const long long k0 = (long long)i * i + (long long)j * j + (long long)k * k;
            if (k0 < (long long)kmax * kmax) {
                so = shell_of(sqrt((double)k0));
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double2 f = F[(3 + q) * N + m];
                    v[5 + q] = sq(f.x / dN) + sq(f.y / dN);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kSpectra; ++q) val[q * kThreads + threadIdx.x] = v[q];
        shell[threadIdx.x] = sk;
        shell[kThreads + threadIdx.x] = so;
        __syncthreads();
        if (threadIdx.x < kSpectra) {  // one thread per spectrum, modes in order
            const int q = threadIdx.x;
            const int *sh = shell + (q < 5 ? 0 : kThreads);
            double *h = hist + q * ks;
            const double *vq = val + q * kThreads;
            for (int t = 0; t < kThreads; ++t)
                if (sh[t] >= 0) h[sh[t]] += vq[t];
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < kSpectra * kmax; t += blockDim.x)
        partials[(size_t)blockIdx.x * kSpectra * kmax + t] = hist[(t / kmax) * ks + t % kmax];
}

__global__ void k_spec_reduce(const double *partials, int nblocks, int n, double *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partials[(size_t)b * n + t];
    out[t] = s;
}

size_t fields_bytes(const BoxParams &p) {
    return sizeof(double2) * kSpectraFields * (size_t)p.N;
}

}  // namespace

size_t spectra_scratch_bytes(const BoxParams &p) {
    const int kmax = spectra_kmax(p);
    return fields_bytes(p) + sizeof(double) * (size_t)kSpecBlocks * kSpectra * kmax;
}

cudaError_t launch_spectra(const BoxDev &b, void *scratch, double *d_out, int *fft_status,
                           cudaStream_t st) {
    const BoxParams &p = b.p;
    const int kmax = spectra_kmax(p);
    double2 *F = static_cast<double2 *>(scratch);
    double *partials = reinterpret_cast<double *>(static_cast<char *>(scratch) + fields_bytes(p));
    *fft_status = CUFFT_SUCCESS;
    k_spec_fields<<<4 * 148, kThreads, 0, st>>>(b, F);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // forward 3-D transforms of the seven fields (x fastest: dims nz, ny, nx)
    cufftHandle plan;
    long long dims[3] = {p.n[2], p.n[1], p.n[0]};
    size_t work = 0;
    cufftResult r = cufftCreate(&plan);
    if (r == CUFFT_SUCCESS) {
        r = cufftMakePlanMany64(plan, 3, dims, nullptr, 1, p.N, nullptr, 1, p.N, CUFFT_Z2Z,
                                kSpectraFields, &work);
        if (r == CUFFT_SUCCESS) r = cufftSetStream(plan, st);
        if (r == CUFFT_SUCCESS)
            r = cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex *>(F),
                             reinterpret_cast<cufftDoubleComplex *>(F), CUFFT_FORWARD);
        e = cudaStreamSynchronize(st);  // the plan's work area outlives the transform
        cufftDestroy(plan);
    }
    if (r != CUFFT_SUCCESS) {
        *fft_status = (int)r;
        return cudaErrorUnknown;
    }
    if (e != cudaSuccess) return e;
    const size_t smem = sizeof(double) * (size_t)kSpectra * (kmax + 1 + kThreads) +
                        sizeof(int) * 2 * kThreads;
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(k_spec_bin, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_spec_bin<<<kSpecBlocks, kThreads, smem, st>>>(F, p.n[0], p.n[1], p.n[2], kmax, partials);
    const int n = kSpectra * kmax;
    k_spec_reduce<<<(n + 127) / 128, 128, 0, st>>>(partials, kSpecBlocks, n, d_out);
    return cudaGetLastError();
}

}  // namespace nuc3d
