"""numpy restatement of postproc::solveFFT (postproc.cpp:931-1184) with the
shell binning of fft::solveShell (fft.cpp:384-572).  TEST INFRASTRUCTURE
ONLY: the checker of the device spectra, never part of the product.

The forward transform follows fft::solveFFT_forward (fft.cpp:182-283):
FFTW_FORWARD sign, normalised by 1/N.  numpy's FFT stands in for FFTW; the
reference's own solveFFT runs in the compiled checker through a DFT stand-in
for FFTW (oracle/ref/fftw_standin.cpp), and this restatement is pinned to it
(tests/test_oracle.py).

Spectra, in this order (the file names solveFFT writes):
  kin, kinc, kins, kinl, kinr  0.5 |.|^2 of the velocity transform, its
      compressive (c) and solenoidal (s) parts and the left/right helical
      halves of s (postproc.cpp:1013-1101), binned by fft.cpp:384-478 over
      the folded wavenumbers with |k| = 1 substituted at k = 0 (so the mean
      flow lands in shell 1);
  hel, ens, den, pre  |f^|^2 of the helicity field w.u, the enstrophy field
      |w|^2/2, density and pressure (postproc.cpp:1132-1184), binned by
      fft.cpp:480-572, which takes kx = i, ky = j, kz = k unfolded and so only
      counts the non-negative octant of wavenumbers.
Shell index: ki = floor(|k|) if frac(|k|) <= 0.5 else floor(|k|) + 1, for
|k| < kmax = min(nx, ny, nz)/2; shells 0 .. kmax-1 are reported.
"""

from __future__ import annotations

import numpy as np

NAMES = ("kin", "kinc", "kins", "kinl", "kinr", "hel", "ens", "den", "pre")

# centraldifference6th.cpp:44-46 / schemes.hpp:38
_CD = (3.0 / 4.0, -3.0 / 20.0, 1.0 / 60.0)


def _cd6(f, axis, h):
    r = lambda o: np.roll(f, -o, axis=axis)  # noqa: E731  f[i + o], periodic
    return (_CD[2] * (r(3) - r(-3)) + _CD[1] * (r(2) - r(-2)) + _CD[0] * (r(1) - r(-1))) / h


def _shell_index(kmag):
    fl = np.floor(kmag)
    return np.where((kmag - fl) - 0.5 <= 0, fl, fl + 1).astype(np.int64)


def _bin(values, kmag, kmax):
    out = np.zeros(kmax + 1)
    on = kmag < kmax
    np.add.at(out, _shell_index(kmag[on]), values[on])
    return out[:kmax]


def spectra(q, dx, dy, dz, gamma, mach):
    """(9, kmax) array of the nine spectra of the conserved state q (5 fields
    shaped (nz, ny, nx)).  Primitives as physicsModel::con2prim with the
    fabs pressure (physicsModel.cpp:324-356)."""
    rho = q[0]
    u, v, w = q[1] / rho, q[2] / rho, q[3] / rho
    p = np.abs((q[4] - 0.5 * rho * (u * u + v * v + w * w)) * (gamma - 1.0))
    nz, ny, nx = rho.shape
    n = nx * ny * nz
    kmax = min(nx, ny, nz) // 2
    # solveQ's fields (postproc.cpp:812-853): vorticity from CD6 gradients
    g = {}
    for name, f in (("u", u), ("v", v), ("w", w)):
        g[name] = (_cd6(f, 2, dx), _cd6(f, 1, dy), _cd6(f, 0, dz))
    w0 = g["w"][1] - g["v"][2]
    w1 = g["u"][2] - g["w"][0]
    w2 = g["v"][0] - g["u"][1]
    ens = (w0 * w0 + w1 * w1 + w2 * w2) * 0.5
    hel = w0 * u + w1 * v + w2 * w

    def fwd(f):
        return np.fft.fftn(f) / n

    U = [fwd(f) for f in (u, v, w)]
    fold = lambda m: np.where(np.arange(m) >= m / 2.0, np.arange(m) - m, np.arange(m))  # noqa: E731
    kx, ky, kz = np.broadcast_arrays(fold(nx)[None, None, :].astype(float),
                                     fold(ny)[None, :, None].astype(float),
                                     fold(nz)[:, None, None].astype(float))
    kmag = np.sqrt(kx * kx + ky * ky + kz * kz)
    kmag = np.where(kmag < 1e-6, 1.0, kmag)
    ku = (kx * U[0] + ky * U[1] + kz * U[2]) / kmag
    s = [U[0] - ku * kx / kmag, U[1] - ku * ky / kmag, U[2] - ku * kz / kmag]
    c = [U[i] - s[i] for i in range(3)]
    # i k x s / |k| (postproc.cpp:1052-1059)
    kxs = [(-(ky * s[2].imag - kz * s[1].imag) + 1j * (ky * s[2].real - kz * s[1].real)) / kmag,
           ((kx * s[2].imag - kz * s[0].imag) - 1j * (kx * s[2].real - kz * s[0].real)) / kmag,
           (-(kx * s[1].imag - ky * s[0].imag) + 1j * (kx * s[1].real - ky * s[0].real)) / kmag]
    r = [0.5 * (s[i] + kxs[i]) for i in range(3)]
    l_ = [0.5 * (s[i] - kxs[i]) for i in range(3)]
    half_e = lambda a: 0.5 * sum(np.abs(x) ** 2 for x in a)  # noqa: E731
    out = [_bin(half_e(a), kmag, kmax) for a in (U, c, s, l_, r)]
    # the unfolded octant binning of fft.cpp:517-531
    ii, jj, kk = np.broadcast_arrays(np.arange(nx)[None, None, :], np.arange(ny)[None, :, None],
                                     np.arange(nz)[:, None, None])
    k0 = ii * ii + jj * jj + kk * kk
    oct_mag = np.where(k0 < kmax * kmax, np.sqrt(k0.astype(float)), float(kmax))
    for f in (hel, ens, rho, p):
        out.append(_bin(np.abs(fwd(f)) ** 2, oct_mag, kmax))
    return np.stack(out)
