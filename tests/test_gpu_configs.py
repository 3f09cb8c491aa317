"""Parity of the plain FP64 path at the benchmark configurations themselves
(C ABI through nuc3d_b200.Solver, against the CPU oracle, which
tests/test_oracle.py pins bitwise to the reference's own translation units).

* Taylor-Green vortex, 64^3, WENO5-JS (eps 1e-6), CD6 viscous terms,
  Lax-Friedrichs split, TVD-RK3 at CFL 0.5, M 0.1, Re 1600, Pr 0.71, 100
  steps (block.cpp:359-395 initial state), with Sutherland viscosity
  (physicsModel.cpp:193-266) and with the power-law model mu = T^0.76 / Re.
  The power-law model is not in the reference: its row is pinned to the
  oracle's restatement only.
* Decaying isotropic turbulence, 256^3, WENO5-Z: the seeded HIT field the
  benchmark advances (seed 0, k_peak 4, turbulent Mach 0.3, Re_lambda 100,
  M 1), one RHS evaluation and one TVD-RK3 step.
* The forced shocklet configuration (turbulent Mach 0.6, band forcing, CFL
  0.4) at 64^3 with the compact schemes in mixed precision: stays finite and
  close to FP64.

Tolerance: per-field relative L2 of 1e-12, as for the small boxes of
tests/test_gpu_step.py.  The oracle runs its lines on all host cores
(NUC3D_ORACLE_THREADS caps them); the 256^3 case holds about 10 GB of host
memory while the oracle runs.
"""

import numpy as np
import pytest

from helpers import desc_from_box, max_rel_l2
from oracle_ctypes import POWERLAW, SUTHERLAND, WENO5JS, WENO5Z, Box, Oracle

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need CUDA"
    return t


@pytest.mark.parametrize("visc", [SUTHERLAND, POWERLAW], ids=["sutherland", "powerlaw"])
def test_taylor_green_64_hundred_steps_match_oracle(torch, visc):
    import nuc3d_b200 as nb
    box = Box(64, 64, 64, scheme=(WENO5JS,) * 3, mach=0.1, reynolds=1600.0, prandtl=0.71,
              visc_model=visc)
    O = Oracle()
    q0 = O.tgv(box)
    with nb.Solver(desc_from_box(box)) as s:
        s.set_state(q0)
        dt, res = s.step(100, 0.5)
        got = s.get_state()
    ref, dt_ref, res_ref = O.run_steps(box, 0.5, 100, [a.copy() for a in q0])
    err = max_rel_l2(got, ref)
    assert err < TOL_FP64, f"64^3 TGV after 100 steps: rel L2 {err:.3e}"
    np.testing.assert_allclose(dt, dt_ref, rtol=1e-12)
    np.testing.assert_allclose(res, res_ref, rtol=1e-9)
    # the flow moved: the state after 100 steps is not the initial state
    assert max_rel_l2(got, q0) > 1e-4


def test_hit_256_rhs_and_one_step_match_oracle(torch):
    import nuc3d_b200 as nb
    desc = nb.BoxDesc(256, 256, 256, mach=1.0, scheme=(nb.WENO5Z,) * 3)
    q, re = nb.hit_field(desc, seed=0, k_peak=4.0, mach_t=0.3, re_lambda=100.0)
    desc.reynolds = re
    box = Box(256, 256, 256, scheme=(WENO5Z,) * 3, mach=desc.mach, reynolds=re,
              prandtl=desc.prandtl, gamma=desc.gamma, t_ref=desc.t_ref, t_inf=desc.t_inf)
    O = Oracle()
    with nb.Solver(desc) as s:
        s.set_state(q)
        out = [torch.zeros(box.shape, dtype=torch.float64, device="cuda") for _ in range(5)]
        dtl = s.rhs(out)
        rhs = [o.cpu().numpy() for o in out]
        del out
        dt, res = s.step(1, 0.5)
        got = s.get_state()
    ref_rhs, dtl_ref = O.rhs(box, q)
    err_rhs = max_rel_l2(rhs, ref_rhs)
    del rhs, ref_rhs
    assert err_rhs < TOL_FP64, f"256^3 HIT RHS: rel L2 {err_rhs:.3e}"
    assert abs(dtl - dtl_ref) <= 1e-14 * dtl_ref
    ref, dt_ref, res_ref = O.run_steps(box, 0.5, 1, [a.copy() for a in q])
    err = max_rel_l2(got, ref)
    assert err < TOL_FP64, f"256^3 HIT after one step: rel L2 {err:.3e}"
    np.testing.assert_allclose(dt, dt_ref, rtol=1e-13)
    np.testing.assert_allclose(res, res_ref, rtol=1e-9)


@pytest.mark.parametrize("scheme,tol", [("crweno5", 1e-6), ("hccs", 1e-3)],
                         ids=["crweno5", "hccs"])
def test_forced_mach06_mixed_compact_schemes_stay_finite(torch, scheme, tol):
    """The forced shocklet configuration at 64^3: seeded HIT at turbulent
    Mach 0.6, band forcing on 0 < |k| <= 2 at the initial dissipation rate,
    CFL 0.4, with CRWENO5 and with hccs (CRWENO5 with the hybrid linear /
    weighted switch) in mixed precision (FP32 line solves).  The mixed run
    stays finite for 500 steps, and after 100 steps it is within `tol`
    (per-field relative L2) of the FP64 run and its kinetic energy within
    1e-4.  hccs's switch is discontinuous: a row that FP32 rounding moves
    across it changes that face by the local flux jump, hence its wider
    bar."""
    import nuc3d_b200 as nb
    sch = nb.CRWENO5 if scheme == "crweno5" else nb.HCCS
    init = {"kind": "hit", "seed": 0, "k_peak": 4.0, "mach_t": 0.6, "re_lambda": 100.0}
    with nb.Solver(nb.BoxDesc(64, 64, 64, mach=1.0)) as s:
        s.init_state(init)
        rate = s.stats()["dissipation"]
    finals, ke = {}, {}
    for prec in (nb.FP64, nb.MIXED):
        d = nb.BoxDesc(64, 64, 64, mach=1.0, scheme=(sch,) * 3, precision=prec,
                       forcing=nb.FORCING_BAND, forcing_amp=rate, forcing_k=2.0)
        with nb.Solver(d) as s:
            s.init_state(init)
            s.step(100, 0.4, stats=False)
            finals[prec] = s.get_state()
            ke[prec] = s.stats()["kinetic"]
            if prec == nb.MIXED:
                for _ in range(4):
                    s.step(100, 0.4, stats=False)
                    s.sync()  # raises on a non-finite state
                q = s.get_state()
                assert all(np.isfinite(a).all() for a in q)
                assert 0.0 < s.stats()["kinetic"] < 1.0
    assert max_rel_l2(finals[nb.MIXED], finals[nb.FP64]) < tol
    assert abs(ke[nb.MIXED] - ke[nb.FP64]) <= 1e-4 * ke[nb.FP64]
