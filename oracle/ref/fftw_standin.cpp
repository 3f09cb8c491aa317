// Definitions for the FFTW stand-in declared in fftw3.h / fftw3-mpi.h.
// TEST INFRASTRUCTURE ONLY.  A plan remembers its length, sign and buffers;
// executing it evaluates the DFT definition directly (O(N^2) per line, fine
// for the checker's box sizes) in long double.
#include "fftw3-mpi.h"

#include <cmath>
#include <cstdlib>
#include <vector>

struct fftw_plan_s {
    int n;
    int sign;
    fftw_complex *in;
    fftw_complex *out;
};

fftw_complex *fftw_alloc_complex(size_t n) {
    return static_cast<fftw_complex *>(std::calloc(n ? n : 1, sizeof(fftw_complex)));
}
void fftw_free(void *p) { std::free(p); }

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned) {
    return new fftw_plan_s{n, sign, in, out};
}

void fftw_destroy_plan(fftw_plan plan) { delete plan; }

void fftw_execute(const fftw_plan p) {
    const int n = p->n;
    const long double two_pi = 6.283185307179586476925286766559005768L;
    std::vector<long double> re(n), im(n);
    for (int k = 0; k < n; ++k) {
        long double sr = 0.0L, si = 0.0L;
        for (int j = 0; j < n; ++j) {
            const long double a = p->sign * two_pi * (long double)((long long)k * j % n) / n;
            const long double c = std::cos(a), s = std::sin(a);
            const long double xr = p->in[j][0], xi = p->in[j][1];
            sr += xr * c - xi * s;
            si += xr * s + xi * c;
        }
        re[k] = sr;
        im[k] = si;
    }
    for (int k = 0; k < n; ++k) {
        p->out[k][0] = (double)re[k];
        p->out[k][1] = (double)im[k];
    }
}

void fftw_mpi_init(void) {}

ptrdiff_t fftw_mpi_local_size_1d(ptrdiff_t n0, MPI_Comm, int, unsigned, ptrdiff_t *local_ni,
                                 ptrdiff_t *local_i_start, ptrdiff_t *local_no,
                                 ptrdiff_t *local_o_start) {
    *local_ni = n0;
    *local_i_start = 0;
    *local_no = n0;
    *local_o_start = 0;
    return n0;
}

fftw_plan fftw_mpi_plan_dft_1d(ptrdiff_t n0, fftw_complex *in, fftw_complex *out, MPI_Comm,
                               int sign, unsigned flags) {
    return fftw_plan_dft_1d((int)n0, in, out, sign, flags);
}
