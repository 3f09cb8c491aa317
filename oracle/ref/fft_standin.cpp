// Stand-in definitions for the reference's nuc3d::fft class (declared in the
// reference's fft.h).  TEST INFRASTRUCTURE ONLY.  The reference's spectral
// routines need FFTW-MPI, which this machine does not have; the hot path under
// test (Forcing None) never calls them, so every method except construction
// and a no-op initFFT stops the checker loudly.
#include "fft.h"

#include <cstdio>
#include <cstdlib>

namespace {
[[noreturn]] void no_fft(const char *what) {
    std::fprintf(stderr, "reference checker: %s needs FFTW, which is not built here\n", what);
    std::exit(96);
}
}  // namespace

nuc3d::fft::fft() {}
nuc3d::fft::~fft() {}
void nuc3d::fft::initFFT(MPIComunicator3d_nonblocking &, int, int, int) {}
void nuc3d::fft::solveFFT_forward(const Field &, Field &, Field &, MPIComunicator3d_nonblocking &) {
    no_fft("fft::solveFFT_forward");
}
void nuc3d::fft::solveFFT_backward(const Field &, const Field &, Field &, Field &,
                                   MPIComunicator3d_nonblocking &) {
    no_fft("fft::solveFFT_backward");
}
void nuc3d::fft::solveShell(const Field &, const Field &, MPIComunicator3d_nonblocking &,
                            std::string, int, double) {
    no_fft("fft::solveShell");
}
void nuc3d::fft::solveShell(const double *, MPIComunicator3d_nonblocking &, std::string, int,
                            double) {
    no_fft("fft::solveShell");
}
