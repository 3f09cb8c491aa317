"""Initial states: the host HIT generator (nuc3d_b200.initial, the restatement
of block::initial_hit, block.cpp:397-551, with counter-based phases) and a
numpy model of the device generator's separable truncated synthesis
(init_kernels.cu), checked against each other on the CPU."""

import math

import numpy as np
import pytest

import nuc3d_b200 as nb
from nuc3d_b200.initial import _wavenumbers, hit_velocity, splitmix_uniform, taylor_microscale


def test_splitmix_known_answer():
    # first output of splitmix64 seeded with 1234567 (published test value)
    z = splitmix_uniform(1234567, np.array([1], dtype=np.uint64))
    assert z[0] == (6457827717110365317 >> 11) / 2.0 ** 53


def test_hit_phases_are_reproducible_and_seeded():
    d = nb.BoxDesc(16, 12, 10, mach=1.0)
    a = hit_velocity(d, seed=5, k_peak=2.0, u_rms=0.2)
    b = hit_velocity(d, seed=5, k_peak=2.0, u_rms=0.2)
    c = hit_velocity(d, seed=6, k_peak=2.0, u_rms=0.2)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert not np.allclose(a[0], c[0])
    urms = math.sqrt(sum(float(np.mean(v * v)) for v in a) / 3.0)
    assert abs(urms - 0.2) < 1e-14


def _axis_modes(n, k_peak):
    kc = min(int(6.5 * k_peak + 1.0), n // 2)
    kmax = kc - 1 if 2 * kc == n else kc
    return np.arange(-kc, kmax + 1)


def device_model(desc, seed, k_peak, u_rms):
    """The device generator's algorithm in numpy: coefficients of the
    retained modes only, separable synthesis z -> y -> x, derivatives with the
    Nyquist wavenumber dropped."""
    nx, ny, nz = desc.nx, desc.ny, desc.nz
    kxs, kys, kzs = (_axis_modes(n, k_peak) for n in (nx, ny, nz))
    KZ, KY, KX = np.meshgrid(kzs, kys, kxs, indexing="ij")
    kx, ky, kz = (K.astype(np.float64) for K in (KX, KY, KZ))
    idx = ((KX % nx) + nx * ((KY % ny) + ny * (KZ % nz))).astype(np.uint64)
    kmag = np.sqrt(kx * kx + ky * ky + kz * kz)
    k12 = np.sqrt(kx * kx + ky * ky)
    kmag = np.where(kmag < 1e-6, 1.0, kmag)
    pie = 4.0 * math.atan(1.0)
    ek = u_rms ** 2 * 16.0 * math.sqrt(2.0 / pie) * (kmag / k_peak) ** 4 / k_peak * np.exp(
        -2.0 * kmag * kmag / k_peak / k_peak)
    amp = np.sqrt(2.0 * ek / kmag / kmag / 4.0 / pie)
    phi = [2.0 * pie * splitmix_uniform(seed, np.uint64(3) * idx + np.uint64(c + 1)) for c in range(3)]
    a = amp * np.exp(1j * phi[0]) * np.cos(phi[2])
    b = amp * np.exp(1j * phi[1]) * np.sin(phi[2])
    small = k12 < 1e-6
    k212 = np.where(small, 1.0, ky / np.where(small, 1.0, k12))
    k112 = np.where(small, 0.0, kx / np.where(small, 1.0, k12))
    C = [k212 * a + k112 * kz / kmag * b, k212 * kz / kmag * b - k112 * a, -k12 / kmag * b]

    def tw(ks, n):
        r = np.mod(np.outer(ks, np.arange(n)), n)
        return np.exp(2j * np.pi * r / n)  # [m, j]

    def dfac(ks, n, L):
        return np.where(2 * np.abs(ks) == n, 0.0, ks * (2 * math.pi / L))

    Tx, Ty, Tz = tw(kxs, nx), tw(kys, ny), tw(kzs, nz)
    fx, fy, fz = dfac(kxs, nx, desc.lx), dfac(kys, ny, desc.ly), dfac(kzs, nz, desc.lz)
    synth = lambda c: np.einsum("zyx,zk,yj,xi->kji", c, Tz, Ty, Tx, optimize=True)  # noqa: E731
    u, v, w = (synth(c).real for c in C)
    ux = synth(C[0] * 1j * fx[None, None, :]).real
    vy = synth(C[1] * 1j * fy[None, :, None]).real
    wz = synth(C[2] * 1j * fz[:, None, None]).real
    n = float(nx * ny * nz)
    s = [float(np.sum(f * f)) for f in (u, v, w, ux, vy, wz)]
    cur = math.sqrt((s[0] / n + s[1] / n + s[2] / n) / 3.0)
    scale = u_rms / cur
    lam = math.sqrt((s[0] + s[1] + s[2]) / (s[3] + s[4] + s[5]))
    return [f * scale for f in (u, v, w)], lam


@pytest.mark.parametrize("shape,k_peak", [((16, 12, 10), 1.0), ((24, 20, 16), 2.0), ((18, 16, 14), 4.0)])
def test_device_synthesis_model_matches_host_fft(shape, k_peak):
    d = nb.BoxDesc(*shape, mach=1.0)
    host = hit_velocity(d, seed=11, k_peak=k_peak, u_rms=0.25)
    dev, lam = device_model(d, 11, k_peak, 0.25)
    for h, m in zip(host, dev):
        assert np.max(np.abs(h - m)) <= 1e-13 * np.max(np.abs(h))
    lam_host, _ = taylor_microscale(d, host)
    assert abs(lam - lam_host) <= 1e-12 * lam_host


def test_truncation_drops_only_negligible_modes():
    # at 64^3 with k_peak 2 the device keeps |k_d| <= 14 of the 32 per axis
    assert len(_axis_modes(64, 2.0)) == 29 and len(_axis_modes(20, 4.0)) == 20
    d = nb.BoxDesc(40, 40, 40, mach=1.0)
    host = hit_velocity(d, seed=3, k_peak=2.0, u_rms=0.3)
    dev, _ = device_model(d, 3, 2.0, 0.3)
    for h, m in zip(host, dev):
        assert np.max(np.abs(h - m)) <= 1e-13 * np.max(np.abs(h))
