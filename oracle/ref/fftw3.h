/* Type-only stand-in for the FFTW3 names that the reference's fft.h declares
 * members with.  TEST INFRASTRUCTURE ONLY: the reference's FFT code (fft.cpp)
 * is not compiled into the checker; fft_standin.cpp supplies the class's
 * methods instead, and the hot path under test never calls them. */
#ifndef NUC3D_REF_FFTW3_STANDIN_H
#define NUC3D_REF_FFTW3_STANDIN_H
#include <cstddef>
typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;
#endif
