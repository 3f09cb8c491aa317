"""Device-generated initial states and the served form (nuc3d_serve_*).

* nuc3d_init_state reproduces the host generators (nuc3d_b200.initial, the
  restatements of block::initial_taylorgreen / initial_hit, block.cpp:359-551).
* A solve served in a mix of other solves (continuous batching: joining and
  leaving the running batch between chunks) ends in exactly the same state as
  the same solve advanced alone.
* Admission respects the device-memory budget and the slot limit, in
  submission order; errors come back per solve."""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import torch
    assert torch.cuda.is_available()
    torch.cuda.init()
    import nuc3d_b200
    return nuc3d_b200


def test_device_tgv_matches_host(nb):
    d = nb.BoxDesc(24, 20, 16, mach=0.1, reynolds=1600.0, prandtl=0.71)
    with nb.Solver(d) as s:
        info = s.init_state("tgv")
        got = s.get_state()
    ref = nb.taylor_green(d)
    for g, r in zip(got, ref):
        assert np.max(np.abs(g - r)) <= 1e-14 * max(1.0, np.max(np.abs(r)))
    assert info["reynolds"] == 1600.0


@pytest.mark.parametrize("shape,k_peak", [((24, 20, 16), 2.0), ((64, 64, 64), 4.0)])
def test_device_hit_matches_host(nb, shape, k_peak):
    d = nb.BoxDesc(*shape, mach=1.0, scheme=(nb.WENO5Z,) * 3)
    init = {"kind": "hit", "seed": 7, "k_peak": k_peak, "mach_t": 0.3, "re_lambda": 100.0}
    with nb.Solver(d) as s:
        info = s.init_state(init)
        got = s.get_state()
    ref, re = nb.hit_field(d, seed=7, k_peak=k_peak, mach_t=0.3, re_lambda=100.0)
    for g, r in zip(got, ref):
        scale = max(np.max(np.abs(r)), 1e-300)
        assert np.max(np.abs(g - r)) <= 1e-12 * scale
    assert abs(info["reynolds"] - re) <= 1e-10 * re
    assert abs(info["u_rms"] - 0.3 / math.sqrt(3.0)) <= 1e-13


def served_mix(nb):
    """(desc, init, nsteps, cfl) of a small mixed stream: every scheme, both
    PDE models, different sizes, seeds, Mach numbers and step counts."""
    JS, Z, CR = nb.WENO5JS, nb.WENO5Z, nb.CRWENO5
    return [
        (nb.BoxDesc(16, 16, 16, scheme=(JS,) * 3, mach=1.0), dict(seed=1, mach_t=0.2), 7, 0.5),
        (nb.BoxDesc(24, 20, 16, scheme=(Z,) * 3, mach=1.0), dict(seed=2, mach_t=0.4), 3, 0.5),
        (nb.BoxDesc(20, 20, 20, scheme=(CR,) * 3, mach=1.0), dict(seed=3, mach_t=0.3), 5, 0.4),
        (nb.BoxDesc(32, 24, 16, scheme=(Z, JS, CR), mach=1.0), dict(seed=4, mach_t=0.5), 9, 0.45),
        (nb.BoxDesc(18, 16, 20, scheme=(Z,) * 3, mach=1.0, pde_model=nb.EULER3D),
         dict(seed=5, mach_t=0.6), 4, 0.5),
        (nb.BoxDesc(40, 32, 24, scheme=(JS,) * 3, mach=1.0), dict(seed=6, mach_t=0.1), 11, 0.5),
    ]


def run_alone(nb, desc, init, nsteps, cfl, precision):
    from dataclasses import replace
    with nb.Solver(replace(desc, precision=precision)) as s:
        s.init_state(init)
        s.step(nsteps, cfl, stats=False)
        s.sync()
        return s.get_state(), s.desc.reynolds


@pytest.mark.parametrize("precision", [0, 1])
def test_served_mix_equals_each_solve_alone(nb, precision):
    mix = served_mix(nb)
    inits = [{"kind": "hit", "k_peak": 4.0, "re_lambda": 60.0, **i} for _, i, _, _ in mix]
    with nb.Server(precision=precision, max_chunk_steps=3, chunk_ms=1.0) as srv:
        tickets = [srv.submit(d, n, cfl, init=init, want_state=True, tag=k)
                   for k, ((d, _, n, cfl), init) in enumerate(zip(mix, inits))]
        results = {r["tag"]: r for r in (srv.wait() for _ in tickets)}
        st = srv.stats()
    assert st["completed"] == len(mix) and st["failed"] == 0
    assert st["peak_resident"] >= 2  # solves overlapped on the device
    for k, ((d, _, n, cfl), init) in enumerate(zip(mix, inits)):
        r = results[k]
        assert r["status"] == nb.OK, r["error"]
        assert r["steps"] == n and r["cells"] == d.cells
        assert r["t_submit"] <= r["t_admit"] <= r["t_done"]
        alone, re = run_alone(nb, d, init, n, cfl, precision)
        assert r["reynolds"] == re
        for a, b in zip(r["state"], alone):
            assert np.array_equal(a, b), f"solve {k} differs alone vs in the mix"


def test_admission_by_budget_and_slots(nb):
    d = nb.BoxDesc(24, 24, 24, scheme=(nb.WENO5Z,) * 3, mach=1.0, precision=nb.MIXED)
    per = d.device_bytes()
    with nb.Server(precision=nb.MIXED, budget_bytes=2 * per + per // 2, max_resident=8,
                   max_chunk_steps=2) as srv:
        ts = [srv.submit(d, 6, init={"kind": "hit", "seed": s, "mach_t": 0.3}) for s in range(5)]
        res = [srv.wait(t) for t in ts]
        st = srv.stats()
    assert all(r["status"] == nb.OK for r in res)
    assert st["peak_resident"] == 2 and st["peak_resident_bytes"] <= 2 * per + per // 2
    admits = [r["t_admit"] for r in res]
    assert admits == sorted(admits)  # submission order
    assert st["cell_updates"] == 5 * 6 * d.cells
    with nb.Server(precision=nb.MIXED, max_resident=1) as srv:
        ts = [srv.submit(d, 2, init="tgv") for _ in range(3)]
        res = [srv.wait(t) for t in ts]
        assert srv.stats()["peak_resident"] == 1
    for a, b in zip(res, res[1:]):
        assert a["t_done"] <= b["t_admit"]  # one slot: strictly one after another


def test_serve_state_input_errors_and_timeout(nb):
    d = nb.BoxDesc(20, 16, 12, scheme=(nb.WENO5JS,) * 3, mach=0.3, reynolds=800.0)
    q0 = nb.taylor_green(d)
    bad = [a.copy() for a in q0]
    bad[4][3, 4, 5] = np.nan
    with nb.Server(precision=nb.FP64, budget_bytes=4 * d.device_bytes()) as srv:
        t_ok = srv.submit(d, 5, 0.5, q0=q0, want_state=True)
        t_nan = srv.submit(d, 3, 0.5, q0=bad)
        with pytest.raises(nb.Nuc3dError) as e:
            srv.submit(nb.BoxDesc(96, 96, 96), 1, init="tgv")
        assert e.value.code == nb.ERR_NOMEM  # larger than the whole budget
        with pytest.raises(nb.Nuc3dError) as e:
            srv.wait(12345)
        assert e.value.code == nb.ERR_INVALID
        r_ok = srv.wait(t_ok)
        r_nan = srv.wait(t_nan)
        t_long = srv.submit(nb.BoxDesc(24, 24, 24, mach=0.3), 1000, init="tgv")
        with pytest.raises(nb.Nuc3dError) as e:
            srv.wait(t_long, timeout=0.0)
        assert e.value.code == nb.ERR_TIMEOUT
        assert srv.wait(t_long)["status"] == nb.OK
    assert r_ok["status"] == nb.OK
    alone, _ = _alone_state(nb, d, q0, 5, 0.5)
    for a, b in zip(r_ok["state"], alone):
        assert np.array_equal(a, b)
    assert r_nan["status"] == nb.ERR_NONFINITE and r_nan["state"] is None


def _alone_state(nb, d, q0, n, cfl):
    with nb.Solver(d) as s:
        s.set_state(q0)
        s.step(n, cfl, stats=False)
        return s.get_state(), None


def test_device_stats_match_reference_and_oracle(nb):
    """nuc3d_stats against the reference's solveQ (golden, 12 printed digits)
    and the oracle (dissipation, not in the reference)."""
    from helpers import golden
    from oracle_ctypes import Box, Oracle, WENO5Z
    z = golden("stats.npz")
    nz, ny, nx = (int(v) for v in z["shape"])
    box = Box(nx, ny, nz, scheme=(WENO5Z,) * 3, mach=float(z["mach"]),
              reynolds=float(z["reynolds"]), prandtl=float(z["prandtl"]))
    d = nb.BoxDesc(nx, ny, nz, scheme=(nb.WENO5Z,) * 3, mach=box.mach, reynolds=box.reynolds,
                   prandtl=box.prandtl)
    q = [np.ascontiguousarray(a) for a in z["q"]]
    with nb.Solver(d) as s:
        s.set_state(q)
        st = s.stats()
    got = np.array([st[k] for k in nb.STAT_NAMES])
    ref = z["stats"]
    # the averages of the nine gradients and three vorticity components are
    # summation noise around 0 (periodic box): compare them on the scale of
    # the gradients themselves
    # (so is the average of Q, a divergence): compare those on the scale of
    # the gradients themselves
    scale = float(ref[18])  # sqrt(<(du_i/dx_i)^2>/3)
    assert np.all(np.abs(got[:12] - ref[:12]) <= 1e-13 * scale)
    assert abs(got[13] - ref[13]) <= 1e-12 * scale * scale
    keep = [12] + list(range(14, 25))
    np.testing.assert_allclose(got[keep], ref[keep], rtol=1e-10)
    o = Oracle().stats(box, q)
    np.testing.assert_allclose(got[25], o[25], rtol=1e-12)


@pytest.mark.parametrize("kf,shape", [(1.0, (24, 20, 16)), (2.0, (32, 32, 32)), (2.6, (20, 24, 28))])
def test_spectral_forcing_matches_restatement(nb, kf, shape):
    """The device shell forcing (AddForcing_Const) against its numpy
    restatement: the RHS with forcing minus the RHS without is the forcing."""
    import torch
    from oracle_ctypes import Oracle
    from forcing_oracle import forcing_terms
    base = nb.BoxDesc(*shape, mach=1.0, reynolds=300.0, scheme=(nb.WENO5Z,) * 3)
    forced = nb.BoxDesc(**{**base.__dict__, "forcing": nb.FORCING_CONST, "forcing_amp": 0.05,
                           "forcing_hel": 0.3, "forcing_k": kf})
    with nb.Solver(base) as s:
        s.init_state({"kind": "hit", "seed": 9, "k_peak": 2.0, "mach_t": 0.3})
        q = s.get_state()
    rhs = {}
    for name, d in (("off", base), ("on", forced)):
        with nb.Solver(d) as s:
            s.set_state(q)
            out = [torch.zeros(d.shape, dtype=torch.float64, device="cuda") for _ in range(5)]
            s.rhs(out)
            rhs[name] = [o.cpu().numpy() for o in out]
    from oracle_ctypes import Box
    prim = Oracle().con2prim(Box(*shape, mach=1.0), q)
    terms, _ = forcing_terms(prim[1], prim[2], prim[3], 0.05, 0.3, kf)
    assert np.array_equal(rhs["on"][0], rhs["off"][0])
    for e in range(1, 5):
        got = rhs["off"][e] - rhs["on"][e]
        scale = np.max(np.abs(terms[e - 1]))
        assert scale > 0
        atol = 1e-12 * max(scale, np.max(np.abs(rhs["off"][e])))
        np.testing.assert_allclose(got, terms[e - 1], rtol=0, atol=atol)


@pytest.mark.parametrize("kf,shape,prec", [(2.0, (32, 32, 32), 0), (1.5, (24, 20, 28), 0),
                                           (2.0, (32, 32, 32), 1)])
def test_band_forcing_matches_restatement(nb, kf, shape, prec):
    """The band forcing at a fixed injection rate (NUC3D_FORCING_BAND) against
    its numpy restatement (forcing_oracle.band_forcing_terms): the RHS with
    forcing minus the RHS without is the forcing, in FP64 and (forcing in
    FP64, RHS in FP32) in mixed precision."""
    import torch
    from oracle_ctypes import Box, Oracle
    from forcing_oracle import band_forcing_terms
    base = nb.BoxDesc(*shape, mach=1.0, reynolds=300.0, scheme=(nb.WENO5Z,) * 3, precision=prec)
    forced = nb.BoxDesc(**{**base.__dict__, "forcing": nb.FORCING_BAND, "forcing_amp": 0.2,
                           "forcing_k": kf})
    with nb.Solver(nb.BoxDesc(*shape, mach=1.0)) as s:
        s.init_state({"kind": "hit", "seed": 4, "k_peak": 2.0, "mach_t": 0.4})
        q = s.get_state()
    rhs = {}
    for name, d in (("off", base), ("on", forced)):
        with nb.Solver(d) as s:
            s.set_state(q)
            out = [torch.zeros(d.shape, dtype=torch.float64, device="cuda") for _ in range(5)]
            s.rhs(out)
            rhs[name] = [o.cpu().numpy() for o in out]
    prim = Oracle().con2prim(Box(*shape, mach=1.0), q)
    terms, (e_b, gain) = band_forcing_terms(prim[1], prim[2], prim[3], 0.2, kf)
    assert e_b > 0 and gain > 0
    assert np.array_equal(rhs["on"][0], rhs["off"][0])
    # FP64: the forcing to 1e-12 of the larger of the forcing and the RHS;
    # mixed: the RHS is held in FP32, so its rounding (1e-7 of the RHS) shows
    rel = 1e-12 if prec == 0 else 3e-7
    for e in range(1, 5):
        got = rhs["off"][e] - rhs["on"][e]
        scale = np.max(np.abs(terms[e - 1]))
        assert scale > 0
        atol = rel * max(scale, np.max(np.abs(rhs["off"][e])))
        np.testing.assert_allclose(got, terms[e - 1], rtol=0, atol=atol)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_spectral_forcing_matches_reference_golden(nb, tag):
    """The device forced RHS against the reference's own (AddForcing_Const run
    by the compiled reference, FFTs through the DFT stand-in for FFTW)."""
    import torch
    from helpers import golden
    z = golden("forcing.npz")
    nz, ny, nx = (int(v) for v in z[f"{tag}_shape"])
    desc = nb.BoxDesc(nx, ny, nz, mach=float(z["mach"]), reynolds=float(z["reynolds"]),
                      prandtl=0.71, scheme=(nb.WENO5Z,) * 3, forcing=nb.FORCING_CONST,
                      forcing_amp=float(z["amp"]), forcing_hel=float(z["hel"]),
                      forcing_k=float(z[f"{tag}_kf"]))
    with nb.Solver(desc) as s:
        s.set_state([np.ascontiguousarray(a) for a in z[f"{tag}_q"]])
        out = [torch.zeros(desc.shape, dtype=torch.float64, device="cuda") for _ in range(5)]
        s.rhs(out)
        got = [o.cpu().numpy() for o in out]
    for e in range(5):
        ref = z[f"{tag}_rhs_on"][e]
        assert np.linalg.norm(got[e] - ref) <= 1e-12 * np.linalg.norm(ref)


def test_spectra_match_reference_golden(nb):
    """nuc3d_spectra (cuFFT transforms, device binning) against the
    reference's own postproc::solveFFT spectra (12 printed digits, FFTs
    through the DFT stand-in for FFTW): all nine spectra, a non-cubic box
    (kmax 5, shell sizes differ per axis) and a 16^3 one; a box in a batch
    gives the same bits as alone."""
    from helpers import golden
    z = golden("spectra.npz")
    for tag in ("a", "b"):
        nz, ny, nx = (int(v) for v in z[f"{tag}_shape"])
        desc = nb.BoxDesc(nx, ny, nz, mach=float(z[f"{tag}_mach"]))
        q = [np.ascontiguousarray(a) for a in z[f"{tag}_q"]]
        with nb.Solver(desc) as s:
            s.set_state(q)
            got = s.spectra()
        ref = z[f"{tag}_spectra"]
        assert got.shape == ref.shape
        np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-13 * np.abs(ref).max())
        with nb.Batch(nb.FP64) as b:
            other = b.add(nb.BoxDesc(24, 20, 16, mach=0.3))
            bid = b.add(desc)
            b.set_state(bid, q)
            b.init_state(other, "tgv")
            assert np.array_equal(b.spectra(bid), got)
