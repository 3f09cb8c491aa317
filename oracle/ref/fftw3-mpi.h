/* See fftw3.h in this directory.  TEST INFRASTRUCTURE ONLY. */
#ifndef NUC3D_REF_FFTW3_MPI_STANDIN_H
#define NUC3D_REF_FFTW3_MPI_STANDIN_H
#include "fftw3.h"
#endif
