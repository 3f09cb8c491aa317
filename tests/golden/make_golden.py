"""Generate the golden fixtures in this directory from the REFERENCE'S OWN
CODE (oracle/_ref/libnuc3d_ref.so, built by ``make -C oracle ref`` from the
reference sources).  Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden.py

The fixtures pin both the C restatement (oracle/) and, through it, the CUDA
path.  Inputs are seeded; every array is FP64 in numpy (nz, ny, nx) order.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "oracle"))

from oracle_ctypes import (AUSM, AUSMP, CD2, CD6, CD8, CRWENO5, HCCS, HCCS77, HCCS78,  # noqa: E402
                           UPWIND1, WENO3JS, WENO5JS, WENO5Z, WENO7, Box, Oracle, Reference)

SCHEME_TAG = {WENO5JS: "js", WENO5Z: "z", CRWENO5: "cr", WENO7: "w7", HCCS: "hc", HCCS77: "h77",
              HCCS78: "h78", WENO3JS: "w3", UPWIND1: "u1"}


def perturbed_tgv(box: Box, seed: int):
    """Taylor-Green state with seeded multiplicative noise (breaks the TGV
    symmetries so that axis or sign slips cannot cancel)."""
    q = Oracle().tgv(box)
    rng = np.random.default_rng(seed)
    return [np.ascontiguousarray(a * (1.0 + 0.02 * rng.standard_normal(a.shape))) for a in q]


def main():
    R = Reference()
    if sys.argv[1:] == ["hccs_siblings"]:  # only the hccs77 / hccs78 fixtures
        hccs_sibling_fixtures(R)
        print("fixtures written to", HERE)
        return
    if sys.argv[1:] == ["low_order"]:  # only the weno3js / upwind1st fixtures
        low_order_fixtures(R)
        print("fixtures written to", HERE)
        return
    if sys.argv[1:] == ["viscous_schemes"]:  # only the cd2 / cd8 fixtures
        viscous_scheme_fixtures(R)
        print("fixtures written to", HERE)
        return
    rng = np.random.default_rng(2024)
    out = {}
    # --- per-operator: reconstruction, CD6, RK stages -------------------
    shape = (5, 4, 14)
    for s in (WENO5JS, WENO5Z, CRWENO5):
        for up in (1, -1):
            f = rng.standard_normal(shape)
            hl = rng.standard_normal(shape[:2] + (3,))
            hr = rng.standard_normal(shape[:2] + (3,))
            tag = f"{SCHEME_TAG[s]}_{'p' if up > 0 else 'm'}"
            out[f"rec_{tag}_in"], out[f"rec_{tag}_hl"], out[f"rec_{tag}_hr"] = f, hl, hr
            out[f"rec_{tag}_out"] = R.reconstruct_field(s, up, f, hl, hr)
    f = rng.standard_normal(shape)
    hl = rng.standard_normal(shape[:2] + (3,))
    hr = rng.standard_normal(shape[:2] + (3,))
    out["cd6_in"], out["cd6_hl"], out["cd6_hr"] = f, hl, hr
    out["cd6_dx"] = np.array(0.37)
    out["cd6_out"] = R.cd6_field(f, 0.37, hl, hr)
    for st in range(3):
        rhs = [rng.standard_normal(40) for _ in range(5)]
        un = [rng.standard_normal(40) for _ in range(5)]
        ui = [rng.standard_normal(40) for _ in range(5)]
        out[f"rk{st}_rhs"], out[f"rk{st}_un"], out[f"rk{st}_ui"] = (np.stack(rhs), np.stack(un),
                                                                    np.stack(ui))
        R.rk3_stage(st, 0.013, rhs, un, ui)
        out[f"rk{st}_out"] = np.stack(ui)
    out["rk_dt"] = np.array(0.013)
    np.savez_compressed(HERE / "operators.npz", **out)

    # --- con2prim + LF split ----------------------------------------------
    box = Box(12, 10, 8, mach=0.3, reynolds=800.0)
    q = perturbed_tgv(box, 7)
    prim, fl, fr, eig = R.split(box, q)
    dirs = ("xi", "eta", "zeta")  # the reference's rotated layouts (euler3d.cpp:71-76)
    np.savez_compressed(HERE / "split.npz", q=np.stack(q), prim=np.stack(prim), eig=eig,
                        **{f"fl_{d}": np.stack(fl[5 * i:5 * i + 5]) for i, d in enumerate(dirs)},
                        **{f"fr_{d}": np.stack(fr[5 * i:5 * i + 5]) for i, d in enumerate(dirs)})

    # --- one RHS and three steps, per scheme, N-S and Euler ----------------
    for s in (WENO5JS, WENO5Z, CRWENO5):
        for ns in (True, False):
            box = Box(16, 12, 10, scheme=(s, s, s), navier_stokes=ns, mach=0.1, reynolds=1600.0,
                      prandtl=0.71)
            q = perturbed_tgv(box, 11 + s)
            rhs, dtl = R.rhs(box, q)
            tag = f"{SCHEME_TAG[s]}_{'ns' if ns else 'eu'}"
            qn, dt, res = R.run_steps(box, 0.5, 3, q)
            np.savez_compressed(HERE / f"step_{tag}.npz", q0=np.stack(q), rhs=np.stack(rhs),
                                dt_local=np.array(dtl), q3=np.stack(qn), dt=dt, res=res,
                                shape=np.array(box.shape), mach=box.mach, reynolds=box.reynolds,
                                prandtl=box.prandtl)

    # --- Taylor-Green 24^3, WENO5-JS + CD6, 10 steps (config-1 physics) ----
    box = Box(24, 24, 24, mach=0.1, reynolds=1600.0, prandtl=0.71)
    q0 = Oracle().tgv(box)
    qn, dt, res = R.run_steps(box, 0.5, 10, q0)
    np.savez_compressed(HERE / "tgv24_js_10.npz", q10=np.stack(qn), dt=dt, res=res)
    stats_fixture(R)
    weno7_fixtures(R)
    ausm_fixtures(R)
    spectra_fixture(R)
    forcing_fixture(R)
    hccs_fixtures(R)
    hccs_sibling_fixtures(R)
    low_order_fixtures(R)
    print("fixtures written to", HERE)


def hccs_fixtures(R):
    """The reference's hccs (hybrid compact scheme; its hccs.cpp compiled with
    an injected declaration of the two names it uses before declaring them):
    both directions on smooth lines (the linear compact rows) and rough ones
    (the weighted rows), 4-wide halos; one RHS plus three steps, N-S and
    Euler."""
    rng = np.random.default_rng(44)
    out = {}
    shape = (5, 4, 20)
    x = np.linspace(0.0, 2.0 * np.pi, shape[2], endpoint=False)
    for up in (1, -1):
        for kind in ("smooth", "rough"):
            if kind == "smooth":
                f = np.sin(x)[None, None, :] + 0.05 * rng.standard_normal(shape)
            else:
                f = rng.standard_normal(shape) * np.exp(rng.standard_normal(shape))
            hl = rng.standard_normal(shape[:2] + (4,))
            hr = rng.standard_normal(shape[:2] + (4,))
            tag = f"hc_{kind}_{'p' if up > 0 else 'm'}"
            out[f"rec_{tag}_in"], out[f"rec_{tag}_hl"], out[f"rec_{tag}_hr"] = f, hl, hr
            out[f"rec_{tag}_out"] = R.reconstruct_field(HCCS, up, f, hl, hr)
    np.savez_compressed(HERE / "operators_hc.npz", **out)
    for ns in (True, False):
        box = Box(16, 12, 10, scheme=(HCCS,) * 3, navier_stokes=ns, mach=0.3, reynolds=800.0,
                  prandtl=0.71)
        q = perturbed_tgv(box, 11 + HCCS)
        rhs, dtl = R.rhs(box, q)
        qn, dt, res = R.run_steps(box, 0.5, 3, q)
        np.savez_compressed(HERE / f"step_hc_{'ns' if ns else 'eu'}.npz", q0=np.stack(q),
                            rhs=np.stack(rhs), dt_local=np.array(dtl), q3=np.stack(qn), dt=dt,
                            res=res, shape=np.array(box.shape), mach=box.mach,
                            reynolds=box.reynolds, prandtl=box.prandtl)


def hccs_sibling_fixtures(R):
    """The reference's hccs77 (WENO7-Z blended into the 7th-order upwind
    compact rows, a tridiagonal line system) and hccs78 (WENO7-Z blended with
    the 8th-order central value, explicit): both directions on smooth and
    rough lines, 4-wide halos; one RHS plus three steps, N-S and Euler."""
    rng = np.random.default_rng(45)
    shape = (5, 4, 20)
    x = np.linspace(0.0, 2.0 * np.pi, shape[2], endpoint=False)
    for sch in (HCCS77, HCCS78):
        out = {}
        for up in (1, -1):
            for kind in ("smooth", "rough"):
                if kind == "smooth":
                    f = np.sin(x)[None, None, :] + 0.05 * rng.standard_normal(shape)
                else:
                    f = rng.standard_normal(shape) * np.exp(rng.standard_normal(shape))
                hl = rng.standard_normal(shape[:2] + (4,))
                hr = rng.standard_normal(shape[:2] + (4,))
                tag = f"{kind}_{'p' if up > 0 else 'm'}"
                out[f"rec_{tag}_in"], out[f"rec_{tag}_hl"], out[f"rec_{tag}_hr"] = f, hl, hr
                out[f"rec_{tag}_out"] = R.reconstruct_field(sch, up, f, hl, hr)
        np.savez_compressed(HERE / f"operators_{SCHEME_TAG[sch]}.npz", **out)
        for ns in (True, False):
            box = Box(16, 12, 10, scheme=(sch,) * 3, navier_stokes=ns, mach=0.3, reynolds=800.0,
                      prandtl=0.71)
            q = perturbed_tgv(box, 11 + sch)
            rhs, dtl = R.rhs(box, q)
            qn, dt, res = R.run_steps(box, 0.5, 3, q)
            np.savez_compressed(HERE / f"step_{SCHEME_TAG[sch]}_{'ns' if ns else 'eu'}.npz",
                                q0=np.stack(q), rhs=np.stack(rhs), dt_local=np.array(dtl),
                                q3=np.stack(qn), dt=dt, res=res, shape=np.array(box.shape),
                                mach=box.mach, reynolds=box.reynolds, prandtl=box.prandtl)


def low_order_fixtures(R):
    """The reference's weno3js (2-cell halos) and upwind1st (1-cell halos):
    both directions on smooth and rough lines; one RHS plus three steps of the
    Euler equations only.  With Navier-Stokes the reference hands its CD6
    viscous stencils these schemes' halo width (2 or 1 cells against the 3
    they read), so its viscous terms read outside their data; no fixture is
    taken from that combination."""
    rng = np.random.default_rng(46)
    shape = (5, 4, 20)
    x = np.linspace(0.0, 2.0 * np.pi, shape[2], endpoint=False)
    for sch, halo in ((WENO3JS, 2), (UPWIND1, 1)):
        out = {}
        for up in (1, -1):
            for kind in ("smooth", "rough"):
                if kind == "smooth":
                    f = np.sin(x)[None, None, :] + 0.05 * rng.standard_normal(shape)
                else:
                    f = rng.standard_normal(shape) * np.exp(rng.standard_normal(shape))
                hl = rng.standard_normal(shape[:2] + (halo,))
                hr = rng.standard_normal(shape[:2] + (halo,))
                tag = f"{kind}_{'p' if up > 0 else 'm'}"
                out[f"rec_{tag}_in"], out[f"rec_{tag}_hl"], out[f"rec_{tag}_hr"] = f, hl, hr
                out[f"rec_{tag}_out"] = R.reconstruct_field(sch, up, f, hl, hr)
        np.savez_compressed(HERE / f"operators_{SCHEME_TAG[sch]}.npz", **out)
        box = Box(16, 12, 10, scheme=(sch,) * 3, navier_stokes=False, mach=0.3, reynolds=800.0,
                  prandtl=0.71)
        q = perturbed_tgv(box, 11 + sch)
        rhs, dtl = R.rhs(box, q)
        qn, dt, res = R.run_steps(box, 0.5, 3, q)
        np.savez_compressed(HERE / f"step_{SCHEME_TAG[sch]}_eu.npz", q0=np.stack(q),
                            rhs=np.stack(rhs), dt_local=np.array(dtl), q3=np.stack(qn), dt=dt,
                            res=res, shape=np.array(box.shape), mach=box.mach,
                            reynolds=box.reynolds, prandtl=box.prandtl)


# (tag, inviscid scheme, differential scheme per direction) of the viscous-
# scheme step fixtures
VIS_STEP_CASES = (("js_cd2", WENO5JS, (CD2, CD2, CD2)), ("w7_cd8", WENO7, (CD8, CD8, CD8)),
                  ("w3_cd2", WENO3JS, (CD2, CD2, CD2)), ("u1_cd2", UPWIND1, (CD2, CD2, CD2)),
                  ("hc_mix", HCCS, (CD8, CD2, CD6)))


def viscous_scheme_fixtures(R):
    """The reference's other differential schemes, centraldifference2nd and
    centraldifference8th (Method.in scheme_*_vis cd2 / cd8): the operators at
    every tilesize they accept (cd8 reads 4 cells, so only tilesize 4), and
    one Navier-Stokes RHS plus three steps with inviscid schemes whose
    bufferSize covers the differential stencil (cd8 with a 4-cell scheme; cd2
    with any, weno3js and upwind1st included), plus solveQ's statistics, whose
    gradients take the same schemes."""
    rng = np.random.default_rng(58)
    shape = (5, 4, 16)
    out = {"dx": np.array(0.37)}
    for name, sch, tiles in (("cd2", CD2, (1, 2, 3, 4)), ("cd6", CD6, (4,)), ("cd8", CD8, (4,))):
        for t in tiles:
            f = rng.standard_normal(shape)
            hl = rng.standard_normal(shape[:2] + (t,))
            hr = rng.standard_normal(shape[:2] + (t,))
            k = f"{name}_t{t}"
            out[f"{k}_in"], out[f"{k}_hl"], out[f"{k}_hr"] = f, hl, hr
            out[f"{k}_out"] = R.cd_field(sch, t, f, 0.37, hl, hr)
    np.savez_compressed(HERE / "operators_vis.npz", **out)
    for tag, sch, vis in VIS_STEP_CASES:
        box = Box(16, 12, 10, scheme=(sch,) * 3, vis=vis, mach=0.3, reynolds=800.0,
                  prandtl=0.71)
        q = perturbed_tgv(box, 17 + sch)
        rhs, dtl = R.rhs(box, q)
        qn, dt, res = R.run_steps(box, 0.5, 3, q)
        np.savez_compressed(HERE / f"step_vis_{tag}.npz", q0=np.stack(q), rhs=np.stack(rhs),
                            dt_local=np.array(dtl), q3=np.stack(qn), dt=dt, res=res,
                            shape=np.array(box.shape), mach=box.mach, reynolds=box.reynolds,
                            prandtl=box.prandtl, scheme=np.array(box.scheme),
                            vis=np.array(vis))
    box = Box(24, 20, 16, scheme=(WENO7,) * 3, vis=(CD8, CD2, CD6), mach=0.3, reynolds=400.0)
    q = perturbed_tgv(box, 5)
    np.savez_compressed(HERE / "stats_vis.npz", q=np.stack(q), stats=R.stats(box, q),
                        shape=np.array(box.shape), mach=box.mach, reynolds=box.reynolds,
                        prandtl=box.prandtl, scheme=np.array(box.scheme), vis=np.array(box.vis))


def forcing_fixture(R):
    """physicsModel::AddForcing_Const (physicsModel.cpp:1368-1641) run by the
    reference itself (FFTs through the DFT stand-in for FFTW): one RHS with
    and without the shell forcing on a perturbed Taylor-Green state with a
    mean flow, for shell radii 1 and 2 (helical part 0.3)."""
    out = {}
    for tag, shape, kf in (("a", (16, 12, 10), 1.0), ("b", (16, 16, 16), 2.0)):
        box = Box(*shape, mach=0.5, reynolds=400.0, scheme=(WENO5Z,) * 3)
        rng = np.random.default_rng(31 + shape[1])
        q = [a * (1 + 0.05 * rng.standard_normal(a.shape))
             for a in Oracle().tgv(box, (0.3, -0.2, 0.1))]
        q[2] = q[2] + 0.05 * q[0]
        off, _ = R.rhs(box, q)
        forced = Box(**{**box.__dict__, "forcing": 1, "forcing_amp": 0.05, "forcing_hel": 0.3,
                        "forcing_k": kf})
        on, _ = R.rhs(forced, q)
        out[f"{tag}_q"] = np.stack(q)
        out[f"{tag}_rhs_off"] = np.stack(off)
        out[f"{tag}_rhs_on"] = np.stack(on)
        out[f"{tag}_shape"] = np.array(box.shape)
        out[f"{tag}_kf"] = kf
    out["mach"], out["reynolds"], out["amp"], out["hel"] = 0.5, 400.0, 0.05, 0.3
    np.savez_compressed(HERE / "forcing.npz", **out)


def spectra_fixture(R):
    """postproc::solveFFT's nine shell spectra (reference, FFTs through the
    DFT stand-in for FFTW) of a perturbed Taylor-Green state with a mean flow
    on a non-cubic box (kmax = 5), and of a 16^3 one."""
    out = {}
    for tag, shape in (("a", (16, 12, 10)), ("b", (16, 16, 16))):
        box = Box(*shape, mach=0.5)
        rng = np.random.default_rng(3 + len(tag) + shape[1])
        q = [a * (1 + 0.05 * rng.standard_normal(a.shape))
             for a in Oracle().tgv(box, (0.3, -0.2, 0.1))]
        q[1] = q[1] + 0.1 * q[0]
        out[f"{tag}_q"] = np.stack(q)
        out[f"{tag}_spectra"] = R.spectra(box, q)
        out[f"{tag}_shape"] = np.array(box.shape)
        out[f"{tag}_mach"] = box.mach
    np.savez_compressed(HERE / "spectra.npz", **out)


def ausm_fixtures(R):
    """The reference's RiemannAUSM / RiemannAUSMp splittings
    (physicsModel.cpp:682-1278): the split fluxes on a box whose local Mach
    number crosses 1 (both branches of the Mach and pressure polynomials), and
    one RHS plus three steps, N-S with WENO5-Z and Euler with WENO5-JS."""
    dirs = ("xi", "eta", "zeta")
    for rm, tag in ((AUSM, "ausm"), (AUSMP, "ausmp")):
        box = Box(12, 10, 8, mach=1.5, reynolds=800.0, riemann=rm)
        q = perturbed_tgv(box, 17 + rm)
        prim, fl, fr, eig = R.split(box, q)
        np.savez_compressed(HERE / f"split_{tag}.npz", q=np.stack(q), eig=eig, mach=box.mach,
                            **{f"fl_{d}": np.stack(fl[5 * i:5 * i + 5]) for i, d in enumerate(dirs)},
                            **{f"fr_{d}": np.stack(fr[5 * i:5 * i + 5]) for i, d in enumerate(dirs)})
        for ns, scheme, mach in ((True, WENO5Z, 1.2), (False, WENO5JS, 0.3)):
            box = Box(16, 12, 10, scheme=(scheme,) * 3, navier_stokes=ns, mach=mach,
                      reynolds=1600.0, prandtl=0.71, riemann=rm)
            q = perturbed_tgv(box, 23 + rm)
            rhs, dtl = R.rhs(box, q)
            qn, dt, res = R.run_steps(box, 0.5, 3, q)
            np.savez_compressed(HERE / f"step_{tag}_{'ns' if ns else 'eu'}.npz", q0=np.stack(q),
                                rhs=np.stack(rhs), dt_local=np.array(dtl), q3=np.stack(qn), dt=dt,
                                res=res, shape=np.array(box.shape), mach=box.mach,
                                reynolds=box.reynolds, prandtl=box.prandtl,
                                scheme=np.array(scheme), riemann=np.array(rm))


def weno7_fixtures(R):
    """The reference's weno7js (bufferSize 4): both reconstruction directions
    with 4-wide halos, and one RHS plus three steps, N-S and Euler."""
    rng = np.random.default_rng(77)
    out = {}
    shape = (5, 4, 14)
    for up in (1, -1):
        f = rng.standard_normal(shape)
        hl = rng.standard_normal(shape[:2] + (4,))
        hr = rng.standard_normal(shape[:2] + (4,))
        tag = f"w7_{'p' if up > 0 else 'm'}"
        out[f"rec_{tag}_in"], out[f"rec_{tag}_hl"], out[f"rec_{tag}_hr"] = f, hl, hr
        out[f"rec_{tag}_out"] = R.reconstruct_field(WENO7, up, f, hl, hr)
    np.savez_compressed(HERE / "operators_w7.npz", **out)
    for ns in (True, False):
        box = Box(16, 12, 10, scheme=(WENO7,) * 3, navier_stokes=ns, mach=0.1, reynolds=1600.0,
                  prandtl=0.71)
        q = perturbed_tgv(box, 11 + WENO7)
        rhs, dtl = R.rhs(box, q)
        qn, dt, res = R.run_steps(box, 0.5, 3, q)
        np.savez_compressed(HERE / f"step_w7_{'ns' if ns else 'eu'}.npz", q0=np.stack(q),
                            rhs=np.stack(rhs), dt_local=np.array(dtl), q3=np.stack(qn), dt=dt,
                            res=res, shape=np.array(box.shape), mach=box.mach,
                            reynolds=box.reynolds, prandtl=box.prandtl)


def stats_fixture(R):
    """postproc::solveQ of the reference (postproc.cpp:736-930) on a perturbed
    non-cubic TGV: the 16 averages of enstrophy.dat and the 9 turb_para.dat
    values (printed by the reference with 12 significant digits)."""
    box = Box(24, 20, 16, scheme=(WENO5Z,) * 3, mach=0.3, reynolds=400.0)
    q = perturbed_tgv(box, 3)
    out = R.stats(box, q)
    np.savez_compressed(HERE / "stats.npz", q=np.stack(q), stats=out,
                        shape=np.array(box.shape), mach=box.mach, reynolds=box.reynolds,
                        prandtl=box.prandtl)
    viscous_scheme_fixtures(R)


if __name__ == "__main__":
    main()
