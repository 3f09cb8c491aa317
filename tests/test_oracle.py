"""The CPU oracle (oracle/nuc3d_oracle.c) pinned against the reference.

Golden fixtures were produced by the reference's own translation units
(tests/golden/make_golden.py); the oracle must reproduce them bitwise.  When
the reference checker library is present (this container), the oracle is
also compared live on fresh seeded inputs.
"""

import numpy as np
import pytest

from helpers import box_from_golden, golden
from oracle_ctypes import (AUSM, AUSMP, CD2, CD6, CD8, CRWENO5, HCCS, HCCS77, HCCS78, LF,
                           QUIRKS_REFERENCE, Q_CRWENO_BOUNDED,
                           Q_WENOZ_BETA2, UPWIND1, WENO3JS, WENO5JS, WENO5Z, WENO7, Box, Oracle,
                           Reference)

TAGS = {WENO5JS: "js", WENO5Z: "z", CRWENO5: "cr"}


@pytest.fixture(scope="module")
def O():
    return Oracle()


@pytest.mark.parametrize("scheme", [WENO5JS, WENO5Z, CRWENO5])
@pytest.mark.parametrize("up", [1, -1])
def test_reconstruct_matches_reference_golden(O, scheme, up):
    z = golden("operators.npz")
    tag = f"{TAGS[scheme]}_{'p' if up > 0 else 'm'}"
    out = O.reconstruct_field(scheme, up, QUIRKS_REFERENCE, z[f"rec_{tag}_in"],
                              z[f"rec_{tag}_hl"], z[f"rec_{tag}_hr"])
    assert np.array_equal(out, z[f"rec_{tag}_out"])


def test_cd6_and_rk3_match_reference_golden(O):
    z = golden("operators.npz")
    out = O.cd6_field(z["cd6_in"], float(z["cd6_dx"]), z["cd6_hl"], z["cd6_hr"])
    assert np.array_equal(out, z["cd6_out"])
    for st in range(3):
        ui = [np.ascontiguousarray(a) for a in z[f"rk{st}_ui"]]
        O.rk3_stage(st, float(z["rk_dt"]), list(z[f"rk{st}_rhs"]), list(z[f"rk{st}_un"]), ui)
        assert np.array_equal(np.stack(ui), z[f"rk{st}_out"])


def test_split_matches_reference_golden(O):
    z = golden("split.npz")
    box = Box(12, 10, 8, mach=0.3, reynolds=800.0)
    q = [np.ascontiguousarray(a) for a in z["q"]]
    prim = O.con2prim(box, q)
    assert np.array_equal(np.stack(prim), z["prim"])


@pytest.mark.parametrize("scheme", [WENO5JS, WENO5Z, CRWENO5])
@pytest.mark.parametrize("ns", [True, False])
def test_rhs_and_steps_match_reference_golden(O, scheme, ns):
    z = golden(f"step_{TAGS[scheme]}_{'ns' if ns else 'eu'}.npz")
    box = box_from_golden(z, scheme, ns)
    q0 = [np.ascontiguousarray(a) for a in z["q0"]]
    rhs, dtl = O.rhs(box, q0)
    assert np.array_equal(np.stack(rhs), z["rhs"])
    assert dtl == float(z["dt_local"])
    q3, dt, res = O.run_steps(box, 0.5, 3, q0)
    assert np.array_equal(np.stack(q3), z["q3"])
    assert np.array_equal(dt, z["dt"]) and np.array_equal(res, z["res"])


def test_tgv24_ten_steps_match_reference_golden(O):
    z = golden("tgv24_js_10.npz")
    box = Box(24, 24, 24, mach=0.1, reynolds=1600.0, prandtl=0.71)
    q, dt, res = O.run_steps(box, 0.5, 10, O.tgv(box))
    assert np.array_equal(np.stack(q), z["q10"])
    assert np.array_equal(dt, z["dt"]) and np.array_equal(res, z["res"])


@pytest.mark.skipif(not Reference.available(), reason="reference checker not built here")
@pytest.mark.parametrize("scheme", [WENO5JS, WENO5Z, CRWENO5])
def test_oracle_matches_reference_live(O, scheme):
    R = Reference()
    rng = np.random.default_rng(99 + scheme)
    box = Box(14, 9, 11, scheme=(scheme,) * 3, mach=0.2, reynolds=500.0)
    q = [a * (1 + 0.05 * rng.standard_normal(a.shape)) for a in O.tgv(box, (0.3, -0.2, 0.1))]
    a, dta = O.rhs(box, q)
    b, dtb = R.rhs(box, q)
    assert np.array_equal(np.stack(a), np.stack(b)) and dta == dtb
    qa, _, ra = O.run_steps(box, 0.4, 2, q)
    qb, _, rb = R.run_steps(box, 0.4, 2, q)
    assert np.array_equal(np.stack(qa), np.stack(qb)) and np.array_equal(ra, rb)


def test_oracle_translation_invariance_without_position_quirks(O):
    """With the two position-dependent reference behaviours switched off
    (WENO5-Z inner beta2, bounded CRWENO lines), the periodic RHS commutes
    with a shift of the box."""
    quirks = QUIRKS_REFERENCE & ~Q_WENOZ_BETA2 & ~Q_CRWENO_BOUNDED
    rng = np.random.default_rng(3)
    for scheme in (WENO5JS, WENO5Z, CRWENO5):
        box = Box(12, 10, 9, scheme=(scheme,) * 3, quirks=quirks, mach=0.3)
        q = [a * (1 + 0.03 * rng.standard_normal(a.shape)) for a in O.tgv(box)]
        r0, _ = O.rhs(box, q)
        qs = [np.ascontiguousarray(np.roll(a, (2, -1, 3), axis=(0, 1, 2))) for a in q]
        r1, _ = O.rhs(box, qs)
        for a, b in zip(r0, r1):
            np.testing.assert_allclose(np.roll(a, (2, -1, 3), axis=(0, 1, 2)), b, rtol=0,
                                       atol=1e-10 * np.abs(a).max())


def test_oracle_weno_z_quirk_changes_only_inner_plus_faces(O):
    rng = np.random.default_rng(5)
    f = rng.standard_normal((2, 3, 16))
    hl = rng.standard_normal((2, 3, 3))
    hr = rng.standard_normal((2, 3, 3))
    a = O.reconstruct_field(WENO5Z, 1, QUIRKS_REFERENCE, f, hl, hr)
    b = O.reconstruct_field(WENO5Z, 1, QUIRKS_REFERENCE & ~Q_WENOZ_BETA2, f, hl, hr)
    diff = np.abs(a - b).max(axis=(0, 1))
    assert np.all(diff[:3] == 0) and np.all(diff[-3:] == 0) and np.all(diff[3:-3] > 0)
    am = O.reconstruct_field(WENO5Z, -1, QUIRKS_REFERENCE, f, hl, hr)
    bm = O.reconstruct_field(WENO5Z, -1, QUIRKS_REFERENCE & ~Q_WENOZ_BETA2, f, hl, hr)
    assert np.array_equal(am, bm)


def test_stats_match_reference_golden(O):
    """postproc::solveQ (postproc.cpp:736-930): the oracle's restatement gives
    the reference's enstrophy.dat averages and turb_para.dat values to the 12
    significant digits the reference prints."""
    z = golden("stats.npz")
    nz, ny, nx = (int(v) for v in z["shape"])
    box = Box(nx, ny, nz, scheme=(WENO5Z,) * 3, mach=float(z["mach"]),
              reynolds=float(z["reynolds"]), prandtl=float(z["prandtl"]))
    got = O.stats(box, list(z["q"]))
    np.testing.assert_allclose(got[:25], z["stats"], rtol=1e-11, atol=0)
    assert got[25] > 0  # dissipation (not in the reference)


@pytest.mark.parametrize("up", [1, -1])
def test_weno7_reconstruct_matches_reference_golden(O, up):
    """The reference's weno7js (Z-form weights, eps 1e-20, 4-wide halos)."""
    z = golden("operators_w7.npz")
    tag = f"w7_{'p' if up > 0 else 'm'}"
    out = O.reconstruct_field(WENO7, up, QUIRKS_REFERENCE, z[f"rec_{tag}_in"], z[f"rec_{tag}_hl"],
                              z[f"rec_{tag}_hr"])
    assert np.array_equal(out, z[f"rec_{tag}_out"])


@pytest.mark.parametrize("ns", [True, False])
def test_weno7_rhs_and_steps_match_reference_golden(O, ns):
    z = golden(f"step_w7_{'ns' if ns else 'eu'}.npz")
    box = box_from_golden(z, WENO7, ns)
    rhs, dtl = O.rhs(box, list(z["q0"]))
    assert np.array_equal(np.stack(rhs), z["rhs"]) and dtl == float(z["dt_local"])
    q3, dt, res = O.run_steps(box, 0.5, 3, list(z["q0"]))
    assert np.array_equal(np.stack(q3), z["q3"])
    assert np.array_equal(dt, z["dt"]) and np.array_equal(res, z["res"])


ROTATE = (lambda a: a, lambda a: a.transpose(2, 0, 1), lambda a: a.transpose(1, 2, 0))


def _check_split(O, box, z):
    q = [np.ascontiguousarray(a) for a in z["q"]]
    _, fl, fr, eig = O.split(box, q)
    for d, name in enumerate(("xi", "eta", "zeta")):
        # the reference stores each direction in its rotated layout (euler3d.cpp:71-76)
        assert np.array_equal(np.stack([ROTATE[d](a) for a in fl[d]]), z[f"fl_{name}"])
        assert np.array_equal(np.stack([ROTATE[d](a) for a in fr[d]]), z[f"fr_{name}"])
    assert np.array_equal(eig, z["eig"])


def test_lf_split_fluxes_match_reference_golden(O):
    _check_split(O, Box(12, 10, 8, mach=0.3, reynolds=800.0), golden("split.npz"))


@pytest.mark.parametrize("riemann,tag", [(AUSM, "ausm"), (AUSMP, "ausmp")])
def test_ausm_split_matches_reference_golden(O, riemann, tag):
    """RiemannAUSM / RiemannAUSMp on a box whose local Mach number spans
    1e-17 .. 17, so both branches of every splitting polynomial are used."""
    z = golden(f"split_{tag}.npz")
    _check_split(O, Box(12, 10, 8, mach=float(z["mach"]), reynolds=800.0, riemann=riemann), z)


def ausm_box(z, ns):
    nz, ny, nx = (int(v) for v in z["shape"])
    return Box(nx, ny, nz, scheme=(int(z["scheme"]),) * 3, navier_stokes=ns,
               mach=float(z["mach"]), reynolds=float(z["reynolds"]),
               prandtl=float(z["prandtl"]), riemann=int(z["riemann"]))


@pytest.mark.parametrize("tag", ["ausm", "ausmp"])
@pytest.mark.parametrize("ns", [True, False])
def test_ausm_rhs_and_steps_match_reference_golden(O, tag, ns):
    z = golden(f"step_{tag}_{'ns' if ns else 'eu'}.npz")
    box = ausm_box(z, ns)
    rhs, dtl = O.rhs(box, list(z["q0"]))
    assert np.array_equal(np.stack(rhs), z["rhs"]) and dtl == float(z["dt_local"])
    q3, dt, res = O.run_steps(box, 0.5, 3, list(z["q0"]))
    assert np.array_equal(np.stack(q3), z["q3"])
    assert np.array_equal(dt, z["dt"]) and np.array_equal(res, z["res"])


@pytest.mark.parametrize("tag", ["a", "b"])
def test_spectra_restatement_matches_reference_golden(tag):
    """The numpy restatement of postproc::solveFFT against the reference's own
    spectra (printed to 12 significant digits): folded kinetic spectra with
    the k = 0 mode in shell 1, and the unfolded-octant scalar spectra."""
    import spectra_oracle as so
    z = golden("spectra.npz")
    nz, ny, nx = (int(v) for v in z[f"{tag}_shape"])
    box = Box(nx, ny, nz, mach=float(z[f"{tag}_mach"]))
    got = so.spectra(list(z[f"{tag}_q"]), box.dx, box.dy, box.dz, box.gamma, box.mach)
    ref = z[f"{tag}_spectra"]
    assert got.shape == ref.shape == (9, min(nx, ny, nz) // 2)
    assert np.all(ref[:5, 0] == 0.0)  # shell 0 of the kinetic spectra never fills
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-13 * np.abs(ref).max())


@pytest.mark.parametrize("tag", ["a", "b"])
def test_forcing_restatement_matches_reference_golden(tag):
    """forcing_oracle.forcing_terms (numpy restatement of AddForcing_Const)
    against the reference's own forced RHS minus its unforced RHS (the
    reference's forcing run through the DFT stand-in for FFTW)."""
    from forcing_oracle import forcing_terms
    z = golden("forcing.npz")
    nz, ny, nx = (int(v) for v in z[f"{tag}_shape"])
    q = list(z[f"{tag}_q"])
    prim = Oracle().con2prim(Box(nx, ny, nz, mach=float(z["mach"])), q)
    terms, _ = forcing_terms(prim[1], prim[2], prim[3], float(z["amp"]), float(z["hel"]),
                             float(z[f"{tag}_kf"]))
    d = z[f"{tag}_rhs_off"] - z[f"{tag}_rhs_on"]
    assert np.array_equal(d[0], np.zeros_like(d[0]))  # no mass source
    for e in range(1, 5):
        scale = np.abs(terms[e - 1]).max()
        assert scale > 0
        assert np.abs(d[e] - terms[e - 1]).max() <= 1e-12 * max(scale, np.abs(z[f"{tag}_rhs_off"][e]).max())


def test_band_forcing_restatement_injects_its_rate():
    """forcing_oracle.band_forcing_terms (the band forcing at a fixed
    injection rate, a model the reference does not have: its parity is pinned
    to this restatement only) checked by its defining properties: the mean
    power <f.u> equals the rate, the force is solenoidal and band-limited
    (0 < |k| <= k_f), and the energy source has zero mean."""
    from forcing_oracle import band_forcing_terms
    rng = np.random.default_rng(5)
    nz, ny, nx = 12, 10, 16
    u, v, w = (rng.standard_normal((nz, ny, nx)) for _ in range(3))
    rate, kf = 0.37, 2.0
    terms, (e_b, gain) = band_forcing_terms(u, v, w, rate, kf)
    f = terms[:3]
    assert abs(np.mean(f[0] * u + f[1] * v + f[2] * w) - rate) <= 1e-13 * rate
    assert abs(np.mean(terms[3])) <= 1e-14 * np.abs(terms[3]).max()
    F = [np.fft.fftn(a) for a in f]
    kx = np.fft.fftfreq(nx, 1.0 / nx)[None, None, :]
    ky = np.fft.fftfreq(ny, 1.0 / ny)[None, :, None]
    kz = np.fft.fftfreq(nz, 1.0 / nz)[:, None, None]
    kx, ky, kz = np.broadcast_arrays(kx, ky, kz)
    kmag = np.sqrt(kx * kx + ky * ky + kz * kz)
    big = max(np.abs(a).max() for a in F)
    outside = (kmag == 0) | (kmag > kf + 1e-9)
    assert all(np.abs(a[outside]).max() <= 1e-12 * big for a in F)
    div = kx * F[0] + ky * F[1] + kz * F[2]
    assert np.abs(div).max() <= 1e-12 * big * kf
    assert e_b > 0 and np.isclose(gain, rate / (2.0 * e_b))


@pytest.mark.parametrize("kind", ["smooth", "rough"])
@pytest.mark.parametrize("up", [1, -1])
def test_hccs_reconstruct_matches_reference_golden(O, kind, up):
    """hccs: WENO7 end faces (eps 1e-40, literal squares), identity rows at
    faces 4 and n-4, hybrid rows (linear upwind compact where theta > 1/2,
    CRWENO5-weighted otherwise) solved by the reference's Thomas sweep."""
    z = golden("operators_hc.npz")
    tag = f"hc_{kind}_{'p' if up > 0 else 'm'}"
    out = O.reconstruct_field(HCCS, up, QUIRKS_REFERENCE, z[f"rec_{tag}_in"], z[f"rec_{tag}_hl"],
                              z[f"rec_{tag}_hr"])
    assert np.array_equal(out, z[f"rec_{tag}_out"])


@pytest.mark.parametrize("ns", [True, False])
def test_hccs_rhs_and_steps_match_reference_golden(O, ns):
    z = golden(f"step_hc_{'ns' if ns else 'eu'}.npz")
    box = box_from_golden(z, HCCS, ns)
    rhs, dtl = O.rhs(box, list(z["q0"]))
    assert np.array_equal(np.stack(rhs), z["rhs"]) and dtl == float(z["dt_local"])
    q3, dt, res = O.run_steps(box, 0.5, 3, list(z["q0"]))
    assert np.array_equal(np.stack(q3), z["q3"])
    assert np.array_equal(dt, z["dt"]) and np.array_equal(res, z["res"])


SIBLING_TAGS = {HCCS77: "h77", HCCS78: "h78"}


@pytest.mark.parametrize("scheme", [HCCS77, HCCS78])
@pytest.mark.parametrize("kind", ["smooth", "rough"])
@pytest.mark.parametrize("up", [1, -1])
def test_hccs_siblings_reconstruct_match_reference_golden(O, scheme, kind, up):
    """hccs77 (WENO7-Z blended into the 7th-order upwind compact rows, WENO7-Z
    end faces and identity rows, the reference's Thomas sweep) and hccs78
    (WENO7-Z blended with the 8th-order central value on faces 4..n-4,
    WENO7-Z at the ends), eps 1e-20 and squares through pow."""
    z = golden(f"operators_{SIBLING_TAGS[scheme]}.npz")
    tag = f"{kind}_{'p' if up > 0 else 'm'}"
    out = O.reconstruct_field(scheme, up, QUIRKS_REFERENCE, z[f"rec_{tag}_in"], z[f"rec_{tag}_hl"],
                              z[f"rec_{tag}_hr"])
    assert np.array_equal(out, z[f"rec_{tag}_out"])


@pytest.mark.parametrize("scheme", [HCCS77, HCCS78])
@pytest.mark.parametrize("ns", [True, False])
def test_hccs_siblings_rhs_and_steps_match_reference_golden(O, scheme, ns):
    z = golden(f"step_{SIBLING_TAGS[scheme]}_{'ns' if ns else 'eu'}.npz")
    box = box_from_golden(z, scheme, ns)
    rhs, dtl = O.rhs(box, list(z["q0"]))
    assert np.array_equal(np.stack(rhs), z["rhs"]) and dtl == float(z["dt_local"])
    q3, dt, res = O.run_steps(box, 0.5, 3, list(z["q0"]))
    assert np.array_equal(np.stack(q3), z["q3"])
    assert np.array_equal(dt, z["dt"]) and np.array_equal(res, z["res"])


LOW_ORDER_TAGS = {WENO3JS: "w3", UPWIND1: "u1"}


@pytest.mark.parametrize("scheme", [WENO3JS, UPWIND1])
@pytest.mark.parametrize("kind", ["smooth", "rough"])
@pytest.mark.parametrize("up", [1, -1])
def test_low_order_reconstruct_match_reference_golden(O, scheme, kind, up):
    """weno3js (eps 1e-6, indicators squared as x*x, weights through pow) and
    upwind1st (the upwind cell), with their 2- and 1-cell halos."""
    z = golden(f"operators_{LOW_ORDER_TAGS[scheme]}.npz")
    tag = f"{kind}_{'p' if up > 0 else 'm'}"
    out = O.reconstruct_field(scheme, up, QUIRKS_REFERENCE, z[f"rec_{tag}_in"], z[f"rec_{tag}_hl"],
                              z[f"rec_{tag}_hr"])
    assert np.array_equal(out, z[f"rec_{tag}_out"])


@pytest.mark.parametrize("scheme", [WENO3JS, UPWIND1])
def test_low_order_euler_rhs_and_steps_match_reference_golden(O, scheme):
    """Euler only: with Navier-Stokes the reference gives its CD6 viscous
    stencils these schemes' 2- or 1-cell halo width, too narrow for the 3
    cells they read, so its viscous terms read outside their data."""
    z = golden(f"step_{LOW_ORDER_TAGS[scheme]}_eu.npz")
    box = box_from_golden(z, scheme, False)
    rhs, dtl = O.rhs(box, list(z["q0"]))
    assert np.array_equal(np.stack(rhs), z["rhs"]) and dtl == float(z["dt_local"])
    q3, dt, res = O.run_steps(box, 0.5, 3, list(z["q0"]))
    assert np.array_equal(np.stack(q3), z["q3"])
    assert np.array_equal(dt, z["dt"]) and np.array_equal(res, z["res"])


def _vis_box(z):
    nz, ny, nx = (int(v) for v in z["shape"])
    return Box(nx, ny, nz, scheme=tuple(int(s) for s in z["scheme"]),
               vis=tuple(int(v) for v in z["vis"]), mach=float(z["mach"]),
               reynolds=float(z["reynolds"]), prandtl=float(z["prandtl"]))


@pytest.mark.parametrize("key", ["cd2_t1", "cd2_t2", "cd2_t3", "cd2_t4", "cd6_t4", "cd8_t4"])
def test_differential_schemes_match_reference_golden(O, key):
    """centraldifference2nd / 6th / 8th at the tilesizes they accept: cells
    within the tilesize of a line end read the halo; cd8's inner cells use its
    two one-sided sums, its boundary cells symmetric differences."""
    z = golden("operators_vis.npz")
    scheme = {"cd2": CD2, "cd6": CD6, "cd8": CD8}[key[:3]]
    out = O.cd_field(scheme, int(key[-1]), z[f"{key}_in"], float(z["dx"]), z[f"{key}_hl"],
                     z[f"{key}_hr"])
    assert np.array_equal(out, z[f"{key}_out"])


@pytest.mark.parametrize("tag", ["js_cd2", "w7_cd8", "w3_cd2", "u1_cd2", "hc_mix"])
def test_viscous_schemes_rhs_and_steps_match_reference_golden(O, tag):
    """Navier-Stokes with Method.in scheme_*_vis cd2 / cd8 (one direction mix
    cd8 / cd2 / cd6): RHS, dt and three steps bitwise."""
    z = golden(f"step_vis_{tag}.npz")
    box = _vis_box(z)
    rhs, dtl = O.rhs(box, list(z["q0"]))
    assert np.array_equal(np.stack(rhs), z["rhs"]) and dtl == float(z["dt_local"])
    q3, dt, res = O.run_steps(box, 0.5, 3, list(z["q0"]))
    assert np.array_equal(np.stack(q3), z["q3"])
    assert np.array_equal(dt, z["dt"]) and np.array_equal(res, z["res"])


def test_stats_with_viscous_schemes_match_reference_golden(O):
    """solveQ's gradients take the operator's differential schemes (cd8, cd2,
    cd6 along x, y, z here)."""
    z = golden("stats_vis.npz")
    box = _vis_box(z)
    got = O.stats(box, list(z["q"]))
    np.testing.assert_allclose(got[:25], z["stats"], rtol=1e-11, atol=0)
