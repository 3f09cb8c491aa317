"""The reference's other differential schemes on the CUDA path: Method.in
scheme_*_vis cd2 (centraldifference2nd.cpp) and cd8 (centraldifference8th
.cpp), per direction, beside the default cd6.

* The `differential` operator (nuc3d_differential) against the reference's
  own outputs, bitwise: the kernel spells the reference's operations in its
  order with correctly rounded intrinsics.
* Navier-Stokes RHS and three steps against the reference's runs where its
  halos cover the stencil (cd8 with a 4-cell inviscid scheme; cd2 with any),
  against the oracle elsewhere (cd8 with a 3-cell scheme: the reference's
  stencil reads outside its halo buffer there; this path's halos are
  periodic whatever the scheme).
* The statistics' gradients take the same schemes (postproc.cpp:2285-2297).
* Mixed precision against FP64."""

import numpy as np
import pytest

from helpers import golden, max_rel_l2
from oracle_ctypes import CD2, CD6, CD8, CRWENO5, WENO5Z, Box, Oracle

from test_gpu_step import gpu_rhs, gpu_steps, rhs_tolerance, step_tolerance, TOL_FP64

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need CUDA"
    return t


def _box(z):
    nz, ny, nx = (int(v) for v in z["shape"])
    return Box(nx, ny, nz, scheme=tuple(int(s) for s in z["scheme"]),
               vis=tuple(int(v) for v in z["vis"]), mach=float(z["mach"]),
               reynolds=float(z["reynolds"]), prandtl=float(z["prandtl"]))


@pytest.mark.parametrize("key", ["cd2_t1", "cd2_t2", "cd2_t3", "cd2_t4", "cd6_t4", "cd8_t4"])
def test_differential_operator_matches_reference_bitwise(torch, key):
    import nuc3d_b200 as nb
    z = golden("operators_vis.npz")
    scheme = {"cd2": nb.CD2, "cd6": nb.CD6, "cd8": nb.CD8}[key[:3]]
    dev = [torch.from_numpy(np.ascontiguousarray(z[f"{key}_{p}"])).cuda()
           for p in ("in", "hl", "hr")]
    out = torch.zeros_like(dev[0])
    nb.differential(scheme, int(key[-1]), float(z["dx"]), *dev, out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), z[f"{key}_out"])


def test_differential_operator_refuses_short_halos(torch):
    """cd8 reads 4 cells and cd6 3: a smaller tilesize is refused."""
    import nuc3d_b200 as nb
    a = torch.zeros((2, 2, 16), dtype=torch.float64, device="cuda")
    h = torch.zeros((2, 2, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(nb.Nuc3dError):
        nb.differential(nb.CD8, 3, 0.1, a, h, h, a.clone())
    with pytest.raises(nb.Nuc3dError):
        nb.differential(nb.CD6, 2, 0.1, a, h[..., :2].contiguous(), h[..., :2].contiguous(),
                        a.clone())


@pytest.mark.parametrize("tag", ["js_cd2", "w7_cd8", "w3_cd2", "u1_cd2", "hc_mix"])
def test_navier_stokes_matches_reference(torch, tag):
    """RHS, dt and three steps against the reference's own runs (weno7js and
    hccs at ten times the oracle's one-ulp sensitivity, as everywhere)."""
    z = golden(f"step_vis_{tag}.npz")
    box = _box(z)
    rhs, dtl = gpu_rhs(torch, box, z["q0"])
    assert max_rel_l2(rhs, z["rhs"]) < rhs_tolerance(box, list(z["q0"]))
    assert abs(dtl - float(z["dt_local"])) <= 1e-14 * float(z["dt_local"])
    q3, dt, res = gpu_steps(box, z["q0"], 3)
    assert max_rel_l2(q3, z["q3"]) < step_tolerance(box, list(z["q0"]), 3)
    np.testing.assert_allclose(dt, z["dt"], rtol=1e-13)
    np.testing.assert_allclose(res, z["res"], rtol=1e-9)


@pytest.mark.parametrize("scheme,vis", [(WENO5Z, (CD8, CD8, CD8)), (CRWENO5, (CD2, CD8, CD6)),
                                        (WENO5Z, (CD6, CD6, CD2))])
def test_navier_stokes_with_three_cell_schemes_match_oracle(torch, scheme, vis):
    """cd8 beside a 3-cell inviscid scheme, where the reference's stencil
    outreaches its halo: against the oracle's periodic restatement, RHS and
    three steps at 1e-12, on a box with extents that are not multiples of the
    32 x 8 tiles."""
    box = Box(36, 20, 14, scheme=(scheme,) * 3, vis=vis, mach=0.3, reynolds=500.0)
    rng = np.random.default_rng(71)
    O = Oracle()
    q = [np.ascontiguousarray(a * (1 + 0.02 * rng.standard_normal(a.shape))) for a in O.tgv(box)]
    ref, dref = O.rhs(box, q)
    got, dgot = gpu_rhs(torch, box, q)
    assert max_rel_l2(got, ref) < TOL_FP64
    q3o, dto, _ = O.run_steps(box, 0.5, 3, q)
    q3g, dtg, _ = gpu_steps(box, q, 3)
    assert max_rel_l2(q3g, q3o) < TOL_FP64
    np.testing.assert_allclose(dtg, dto, rtol=1e-13)


def test_statistics_take_the_differential_schemes(torch):
    """solveQ with cd8 / cd2 / cd6 gradients against the reference's printed
    values (12 digits)."""
    import nuc3d_b200 as nb
    z = golden("stats_vis.npz")
    box = _box(z)
    d = nb.BoxDesc(box.nx, box.ny, box.nz, scheme=box.scheme, vis_scheme=box.vis, mach=box.mach,
                   reynolds=box.reynolds, prandtl=box.prandtl)
    with nb.Solver(d) as s:
        s.set_state([np.ascontiguousarray(a) for a in z["q"]])
        st = s.stats()
    got = np.array([st[k] for k in nb.STAT_NAMES])
    ref = z["stats"]
    scale = float(ref[18])
    assert np.all(np.abs(got[:12] - ref[:12]) <= 1e-13 * scale)
    assert abs(got[13] - ref[13]) <= 1e-12 * scale * scale
    keep = [12] + list(range(14, 25))
    np.testing.assert_allclose(got[keep], ref[keep], rtol=1e-10)


def test_mixed_precision_close_to_fp64(torch):
    """cd8 everywhere with WENO5-Z, FP32 bulk against FP64: decaying
    turbulence at 64^3, 50 steps."""
    import nuc3d_b200 as nb
    init = {"kind": "hit", "seed": 4, "k_peak": 4.0, "mach_t": 0.3, "re_lambda": 100.0}
    out = []
    for precision in (nb.FP64, nb.MIXED):
        d = nb.BoxDesc(64, 64, 64, mach=1.0, scheme=(nb.WENO5Z,) * 3,
                       vis_scheme=(nb.CD8, nb.CD8, nb.CD2), precision=precision)
        with nb.Solver(d) as s:
            s.init_state(init)
            s.step(50, 0.5, stats=False)
            out.append(s.get_state())
    err = max_rel_l2(out[1], out[0])
    print(f"cd8/cd8/cd2 mixed vs fp64 after 50 steps: max per-field rel L2 = {err:.3e}")
    assert err < 1e-6
