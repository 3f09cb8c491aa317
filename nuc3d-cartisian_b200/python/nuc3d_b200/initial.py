"""Initial states for the periodic box (host, FP64, numpy).

* ``taylor_green`` restates block::initial_taylorgreen (block.cpp:359-395)
  on the cell centres of block::getXYZ (block.cpp:103-124) for one rank.
* ``hit_field`` restates block::initial_hit (block.cpp:397-551): a
  random-phase solenoidal velocity field with
  E(k) = u_rms^2 * 16 sqrt(2/pi) (k/kp)^4 / kp * exp(-2 (k/kp)^2), built by
  the Craya-Herring projection and an unnormalised backward FFT, rescaled to
  the target rms velocity.  The reference draws its phases from an unseeded
  std::random_device + mt19937 (three per mode, in index order); here phase c
  of the mode at FFT index idx is the splitmix64 output number 3*idx + c + 1
  of the stream seeded with `seed` (Steele, Lea & Flood, "Fast splittable
  pseudorandom number generators", OOPSLA 2014), mapped to [0, 2 pi).  A
  counter-based stream lets the device generator draw the same phases in any
  order, so the host and device fields agree to rounding; like the
  reference's field, neither is pinned to the reference's own draws.
"""

from __future__ import annotations

import math

import numpy as np


def cell_centres(desc, origin=(0.0, 0.0, 0.0)):
    dx, dy, dz = desc.lx / desc.nx, desc.ly / desc.ny, desc.lz / desc.nz
    x = 0.0 + dx * (0.5 + np.arange(desc.nx)) - origin[0]
    y = 0.0 + dy * (0.5 + np.arange(desc.ny)) - origin[1]
    z = 0.0 + dz * (0.5 + np.arange(desc.nz)) - origin[2]
    return np.meshgrid(z, y, x, indexing="ij")[::-1]  # X, Y, Z shaped (nz, ny, nx)


def taylor_green(desc, origin=(0.0, 0.0, 0.0)):
    """Conserved state [rho, rho u, rho v, rho w, rho E] of the TGV."""
    X, Y, Z = cell_centres(desc, origin)
    g, M = desc.gamma, desc.mach
    rho0 = np.ones_like(X)
    u0 = np.sin(X) * np.cos(Y) * np.cos(Z)
    v0 = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w0 = np.zeros_like(X)
    p0 = 1.0 / (g * M * M) + ((np.cos(2.0 * Z) + 2.0) * (np.cos(2.0 * X) + np.cos(2.0 * Y)) - 2.0) / 16.0
    rhoE = p0 / (g - 1.0) + 0.5 * rho0 * (u0 * u0 + v0 * v0 + w0 * w0)
    return [np.ascontiguousarray(a) for a in (rho0, rho0 * u0, rho0 * v0, rho0 * w0, rhoE)]


_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix_uniform(seed, n):
    """Uniform [0, 1) doubles: output number n (uint64 array, n >= 1) of the
    splitmix64 stream seeded with `seed`, top 53 bits."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.asarray(n, dtype=np.uint64) * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _wavenumbers(n):
    k = np.arange(n, dtype=np.float64)
    return np.where(k >= n / 2.0, k - n, k)  # block.cpp:472-474


def hit_velocity(desc, seed=0, k_peak=4.0, u_rms=0.1):
    """Solenoidal random-phase velocity (u, v, w), each (nz, ny, nx)."""
    kx = _wavenumbers(desc.nx)[None, None, :]
    ky = _wavenumbers(desc.ny)[None, :, None]
    kz = _wavenumbers(desc.nz)[:, None, None]
    kx, ky, kz = np.broadcast_arrays(kx, ky, kz)
    kmag = np.sqrt(kx * kx + ky * ky + kz * kz)
    k12 = np.sqrt(kx * kx + ky * ky)
    kmag = np.where(kmag < 1e-6, 1.0, kmag)
    pie = 4.0 * math.atan(1.0)
    ek = u_rms ** 2 * 16.0 * math.sqrt(2.0 / pie) * (kmag / k_peak) ** 4 / k_peak * np.exp(
        -2.0 * kmag * kmag / k_peak / k_peak)
    idx = np.arange(kmag.size, dtype=np.uint64).reshape(kmag.shape)  # i + nx (j + ny k)
    phi = np.stack([2.0 * pie * splitmix_uniform(seed, np.uint64(3) * idx + np.uint64(c + 1))
                    for c in range(3)])
    amp = np.sqrt(2.0 * ek / kmag / kmag / 4.0 / pie)
    a = amp * np.exp(1j * phi[0]) * np.cos(phi[2])
    b = amp * np.exp(1j * phi[1]) * np.sin(phi[2])
    small = k12 < 1e-6
    k212 = np.where(small, 1.0, ky / np.where(small, 1.0, k12))
    k112 = np.where(small, 0.0, kx / np.where(small, 1.0, k12))
    uh = k212 * a + k112 * kz / kmag * b
    vh = k212 * kz / kmag * b - k112 * a
    wh = -k12 / kmag * b
    # unnormalised backward transform; only the real part is kept (block.cpp:504-510)
    n = desc.cells
    vel = [np.ascontiguousarray(np.fft.ifftn(h).real * n) for h in (uh, vh, wh)]
    cur = math.sqrt(sum(float(np.mean(v * v)) for v in vel) / 3.0)
    scale = u_rms / cur
    return [v * scale for v in vel]


def taylor_microscale(desc, vel):
    """lambda = sqrt(<u_i u_i>/3 / <(du_i/dx_i)^2>/3) as postproc.cpp:871,
    with spectral derivatives."""
    kx = _wavenumbers(desc.nx) * (2 * math.pi / desc.lx)
    ky = _wavenumbers(desc.ny) * (2 * math.pi / desc.ly)
    kz = _wavenumbers(desc.nz) * (2 * math.pi / desc.lz)
    ux = np.fft.ifft(1j * kx[None, None, :] * np.fft.fft(vel[0], axis=2), axis=2).real
    vy = np.fft.ifft(1j * ky[None, :, None] * np.fft.fft(vel[1], axis=1), axis=1).real
    wz = np.fft.ifft(1j * kz[:, None, None] * np.fft.fft(vel[2], axis=0), axis=0).real
    u2 = sum(float(np.mean(v * v)) for v in vel) / 3.0
    d2 = (float(np.mean(ux * ux)) + float(np.mean(vy * vy)) + float(np.mean(wz * wz))) / 3.0
    return math.sqrt(u2 / d2), math.sqrt(u2)


def hit_field(desc, seed=0, k_peak=4.0, mach_t=0.3, re_lambda=None):
    """Conserved state of decaying isotropic turbulence with uniform rho = 1,
    p = 1/(gamma M^2) (block.cpp:536-546).  mach_t = sqrt(3) u_rms / c with
    c = 1/M; the reference's u_rms = Mt/M^2/sqrt(3) (block.cpp:422) coincides
    at M = 1.  If re_lambda is given, returns the Reynolds number that gives
    that Re_lambda (postproc.cpp:871-872) as the second value."""
    g, M = desc.gamma, desc.mach
    c = 1.0 / M
    u_rms = mach_t * c / math.sqrt(3.0)
    u, v, w = hit_velocity(desc, seed, k_peak, u_rms)
    rho = np.ones(desc.shape)
    p0 = 1.0 / (g * M * M)
    rhoE = p0 / (g - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    q = [np.ascontiguousarray(a) for a in (rho, rho * u, rho * v, rho * w, rhoE)]
    if re_lambda is None:
        return q
    lam, urms = taylor_microscale(desc, (u, v, w))
    return q, re_lambda / (urms * lam)
