/* Single-process stand-in for the subset of FFTW3's API that the reference's
 * fft.cpp calls.  TEST INFRASTRUCTURE ONLY.  FFTW (an external library the
 * reference links without a pinned version) is not on this machine; the
 * plans here evaluate the published definition of the 1-D DFT,
 *   X_k = sum_n x_n exp(sign * 2 pi i k n / N),  sign = FFTW_FORWARD (-1)
 *         or FFTW_BACKWARD (+1), unnormalised (FFTW's convention),
 * directly in long double with twiddles reduced modulo N, so its results are
 * within a few FP64 ulps of any correct FFT. */
#ifndef NUC3D_REF_FFTW3_STANDIN_H
#define NUC3D_REF_FFTW3_STANDIN_H
#include <cstddef>

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_complex *fftw_alloc_complex(size_t n);
void fftw_free(void *p);
void fftw_execute(const fftw_plan plan);
void fftw_destroy_plan(fftw_plan plan);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
#endif
