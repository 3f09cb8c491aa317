/* See fftw3.h in this directory.  TEST INFRASTRUCTURE ONLY.  The single-rank
 * MPI stand-in (mpi.h) has one process, so a distributed 1-D plan is a local
 * plan over the whole line. */
#ifndef NUC3D_REF_FFTW3_MPI_STANDIN_H
#define NUC3D_REF_FFTW3_MPI_STANDIN_H
#include "fftw3.h"
#include "mpi.h"

void fftw_mpi_init(void);
ptrdiff_t fftw_mpi_local_size_1d(ptrdiff_t n0, MPI_Comm comm, int sign, unsigned flags,
                                 ptrdiff_t *local_ni, ptrdiff_t *local_i_start,
                                 ptrdiff_t *local_no, ptrdiff_t *local_o_start);
fftw_plan fftw_mpi_plan_dft_1d(ptrdiff_t n0, fftw_complex *in, fftw_complex *out, MPI_Comm comm,
                               int sign, unsigned flags);
#endif
