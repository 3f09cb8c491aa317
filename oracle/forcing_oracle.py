"""numpy restatement of physicsModel::AddForcing_Const (physicsModel.cpp:1368-
1641), the spectral shell forcing.  TEST INFRASTRUCTURE ONLY: the checker of
the device forcing, never part of the product.

The reference transforms with FFTW (fft.cpp:182-572: forward normalised by
1/N, backward unnormalised).  FFTW is absent here; the compiled reference runs
its own AddForcing_Const through a DFT stand-in for FFTW
(oracle/ref/fftw_standin.cpp), and this restatement, with numpy's FFTs under
the same conventions, is pinned to it (tests/test_oracle.py, golden
forcing.npz: agreement to ~1e-14 of the forcing's scale).
"""

from __future__ import annotations

import numpy as np


def _wavenumbers(n):
    k = np.arange(n, dtype=np.float64)
    return np.where(k >= n / 2.0, k - n, k)  # physicsModel.cpp:1473-1475


def forcing_terms(u, v, w, amp, hel, kf):
    """The amounts AddForcing_Const subtracts from RHS[1..4] for velocity
    fields u, v, w (each (nz, ny, nx)), and (E_s, E_c, theta)."""
    nz, ny, nx = u.shape
    n = nx * ny * nz
    U = [np.fft.fftn(f) / n for f in (u, v, w)]  # fft.cpp:277-278
    kx = _wavenumbers(nx)[None, None, :]
    ky = _wavenumbers(ny)[None, :, None]
    kz = _wavenumbers(nz)[:, None, None]
    kx, ky, kz = np.broadcast_arrays(kx, ky, kz)
    kmag0 = np.sqrt(kx * kx + ky * ky + kz * kz)
    kmag = np.where(kmag0 < 1e-6, 1.0, kmag0)
    ku = (kx * U[0] + ky * U[1] + kz * U[2]) / kmag
    s = [U[0] - ku * kx / kmag, U[1] - ku * ky / kmag, U[2] - ku * kz / kmag]
    c = [U[i] - s[i] for i in range(3)]
    # helical term (physicsModel.cpp:1512-1526): i k x s / |k|
    kxu0 = (-(ky * s[2].imag - kz * s[1].imag) + 1j * (ky * s[2].real - kz * s[1].real)) / kmag
    kxu1 = ((kx * s[2].imag - kz * s[0].imag) - 1j * (kx * s[2].real - kz * s[0].real)) / kmag
    kxu2 = (-(kx * s[1].imag - ky * s[0].imag) + 1j * (kx * s[1].real - ky * s[0].real)) / kmag
    s = [s[0] + hel * kxu0, s[1] + hel * kxu1, s[2] + hel * kxu2]
    shell = np.abs(kmag - kf) < 0.5
    e_s = float(np.sum(0.5 * sum(np.abs(a) ** 2 for a in s)[shell]))
    e_c = float(np.sum(0.5 * sum(np.abs(a) ** 2 for a in c)[shell]))
    theta = np.sqrt(abs(amp - e_c) / e_s)
    on = np.abs(kmag0 - kf) < 0.5  # second loop: kmag not substituted at k = 0
    F = [np.where(on, a * (theta - 1.0), 0.0) for a in s]
    f = [np.fft.ifftn(a).real * n for a in F]  # backward, unnormalised, real part
    fu = f[0] * u + f[1] * v + f[2] * w  # rho0 = 1
    a_aver = float(np.mean(fu))
    return [f[0], f[1], f[2], fu - a_aver], (e_s, e_c, float(theta))


def band_forcing_terms(u, v, w, rate, kf):
    """The amounts the band forcing at a fixed injection rate subtracts from
    RHS[1..4] (NUC3D_FORCING_BAND, this library's own model: the reference
    has only the shell forcing above), and (E_b, gain).  The solenoidal part
    s of every mode with 0 < |k| <= kf is forced as f = s * rate / (2 E_b),
    E_b = sum over the band of |s|^2 / 2; in physical space with the shell
    forcing's conventions (density 1, energy equation f.u - <f.u>)."""
    nz, ny, nx = u.shape
    n = nx * ny * nz
    U = [np.fft.fftn(f) / n for f in (u, v, w)]
    kx = _wavenumbers(nx)[None, None, :]
    ky = _wavenumbers(ny)[None, :, None]
    kz = _wavenumbers(nz)[:, None, None]
    kx, ky, kz = np.broadcast_arrays(kx, ky, kz)
    kmag0 = np.sqrt(kx * kx + ky * ky + kz * kz)
    kmag = np.where(kmag0 < 1e-6, 1.0, kmag0)
    ku = (kx * U[0] + ky * U[1] + kz * U[2]) / kmag
    s = [U[0] - ku * kx / kmag, U[1] - ku * ky / kmag, U[2] - ku * kz / kmag]
    band = (kmag0 > 0.0) & (kmag0 <= kf + 1e-12)
    e_b = float(np.sum(0.5 * sum(np.abs(a) ** 2 for a in s)[band]))
    gain = rate / (2.0 * e_b) if e_b > 0.0 else 0.0
    F = [np.where(band, a * gain, 0.0) for a in s]
    f = [np.fft.ifftn(a).real * n for a in F]
    fu = f[0] * u + f[1] * v + f[2] * w
    return [f[0], f[1], f[2], fu - float(np.mean(fu))], (e_b, gain)
