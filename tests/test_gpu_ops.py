"""Per-operator parity of the CUDA path (through the C ABI) against the
reference's own outputs (golden fixtures) and the CPU oracle.

Tolerance: single-operator FP64 results agree with the reference to a
relative 1e-13 (the CUDA kernels use FMA contraction and a single-division
weight normalisation, exact rearrangements that round differently)."""

import numpy as np
import pytest

from helpers import golden, rel_l2
from oracle_ctypes import (HCCS, HCCS77, HCCS78, QUIRKS_REFERENCE, Q_WENOZ_BETA2, UPWIND1, WENO3JS,
                           WENO7, Oracle)

pytestmark = pytest.mark.gpu

TOL_OP = 1e-13


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    return torch


def to_dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("scheme", [0, 1, 2])
@pytest.mark.parametrize("up", [1, -1])
def test_reconstruct_golden(torch_cuda, scheme, up):
    import nuc3d_b200 as nb
    torch = torch_cuda
    z = golden("operators.npz")
    tag = f"{['js', 'z', 'cr'][scheme]}_{'p' if up > 0 else 'm'}"
    fin = to_dev(torch, z[f"rec_{tag}_in"])
    out = torch.zeros(fin.shape[:2] + (fin.shape[2] + 1,), dtype=torch.float64, device="cuda")
    nb.reconstruct(scheme, up, QUIRKS_REFERENCE, fin, to_dev(torch, z[f"rec_{tag}_hl"]),
                   to_dev(torch, z[f"rec_{tag}_hr"]), out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), z[f"rec_{tag}_out"]) < TOL_OP


@pytest.mark.parametrize("scheme", [0, 1, 2])
@pytest.mark.parametrize("up", [1, -1])
@pytest.mark.parametrize("quirks", [QUIRKS_REFERENCE, QUIRKS_REFERENCE & ~Q_WENOZ_BETA2])
def test_reconstruct_vs_oracle_larger(torch_cuda, scheme, up, quirks):
    import nuc3d_b200 as nb
    torch = torch_cuda
    rng = np.random.default_rng(10 * scheme + up + 3)
    shape = (7, 9, 61)
    f = rng.standard_normal(shape) * np.exp(rng.standard_normal(shape))  # rough data
    hl = rng.standard_normal(shape[:2] + (3,))
    hr = rng.standard_normal(shape[:2] + (3,))
    ref = Oracle().reconstruct_field(scheme, up, quirks, f, hl, hr)
    out = torch.zeros(shape[:2] + (shape[2] + 1,), dtype=torch.float64, device="cuda")
    nb.reconstruct(scheme, up, quirks, to_dev(torch, f), to_dev(torch, hl), to_dev(torch, hr), out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref) < TOL_OP


@pytest.mark.parametrize("up", [1, -1])
def test_weno7_reconstruct_golden(torch_cuda, up):
    """weno7js with its 4-cell halos against the reference's own outputs."""
    import nuc3d_b200 as nb
    torch = torch_cuda
    z = golden("operators_w7.npz")
    tag = f"w7_{'p' if up > 0 else 'm'}"
    fin = to_dev(torch, z[f"rec_{tag}_in"])
    out = torch.zeros(fin.shape[:2] + (fin.shape[2] + 1,), dtype=torch.float64, device="cuda")
    nb.reconstruct(WENO7, up, QUIRKS_REFERENCE, fin, to_dev(torch, z[f"rec_{tag}_hl"]),
                   to_dev(torch, z[f"rec_{tag}_hr"]), out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), z[f"rec_{tag}_out"]) < TOL_OP


@pytest.mark.parametrize("up", [1, -1])
def test_weno7_reconstruct_vs_oracle_larger(torch_cuda, up):
    """Rough data (values spread over decades, so the Z weights switch) on
    lines of 61 cells."""
    import nuc3d_b200 as nb
    torch = torch_cuda
    rng = np.random.default_rng(70 + up)
    shape = (7, 9, 61)
    f = rng.standard_normal(shape) * np.exp(rng.standard_normal(shape))
    hl = rng.standard_normal(shape[:2] + (4,))
    hr = rng.standard_normal(shape[:2] + (4,))
    ref = Oracle().reconstruct_field(WENO7, up, QUIRKS_REFERENCE, f, hl, hr)
    out = torch.zeros(shape[:2] + (shape[2] + 1,), dtype=torch.float64, device="cuda")
    nb.reconstruct(WENO7, up, QUIRKS_REFERENCE, to_dev(torch, f), to_dev(torch, hl),
                   to_dev(torch, hr), out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), ref) < TOL_OP


@pytest.mark.parametrize("kind", ["smooth", "rough"])
@pytest.mark.parametrize("up", [1, -1])
def test_hccs_reconstruct_golden(torch_cuda, kind, up):
    """hccs (hybrid compact) with 4-cell halos against the reference's own
    outputs; 1e-12 (the blend switches on a threshold and the Z weights use
    eps 1e-40, so the scheme amplifies rounding more than WENO5)."""
    import nuc3d_b200 as nb
    torch = torch_cuda
    z = golden("operators_hc.npz")
    tag = f"hc_{kind}_{'p' if up > 0 else 'm'}"
    fin = to_dev(torch, z[f"rec_{tag}_in"])
    out = torch.zeros(fin.shape[:2] + (fin.shape[2] + 1,), dtype=torch.float64, device="cuda")
    nb.reconstruct(HCCS, up, QUIRKS_REFERENCE, fin, to_dev(torch, z[f"rec_{tag}_hl"]),
                   to_dev(torch, z[f"rec_{tag}_hr"]), out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), z[f"rec_{tag}_out"]) < 1e-12


@pytest.mark.parametrize("scheme,tag", [(HCCS77, "h77"), (HCCS78, "h78")])
@pytest.mark.parametrize("kind", ["smooth", "rough"])
@pytest.mark.parametrize("up", [1, -1])
def test_hccs_siblings_reconstruct_golden(torch_cuda, scheme, tag, kind, up):
    """hccs77 (WENO7-Z blended into 7th-order upwind compact rows, a line
    solve) and hccs78 (WENO7-Z blended with the 8th-order central value) with
    4-cell halos against the reference's own outputs at 1e-12."""
    import nuc3d_b200 as nb
    torch = torch_cuda
    z = golden(f"operators_{tag}.npz")
    key = f"{kind}_{'p' if up > 0 else 'm'}"
    fin = to_dev(torch, z[f"rec_{key}_in"])
    out = torch.zeros(fin.shape[:2] + (fin.shape[2] + 1,), dtype=torch.float64, device="cuda")
    nb.reconstruct(scheme, up, QUIRKS_REFERENCE, fin, to_dev(torch, z[f"rec_{key}_hl"]),
                   to_dev(torch, z[f"rec_{key}_hr"]), out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), z[f"rec_{key}_out"]) < 1e-12


@pytest.mark.parametrize("scheme,tag", [(WENO3JS, "w3"), (UPWIND1, "u1")])
@pytest.mark.parametrize("kind", ["smooth", "rough"])
@pytest.mark.parametrize("up", [1, -1])
def test_low_order_reconstruct_golden(torch_cuda, scheme, tag, kind, up):
    """weno3js (2-cell halos) and upwind1st (1-cell halos) against the
    reference's own outputs at 1e-12."""
    import nuc3d_b200 as nb
    torch = torch_cuda
    z = golden(f"operators_{tag}.npz")
    key = f"{kind}_{'p' if up > 0 else 'm'}"
    fin = to_dev(torch, z[f"rec_{key}_in"])
    out = torch.zeros(fin.shape[:2] + (fin.shape[2] + 1,), dtype=torch.float64, device="cuda")
    nb.reconstruct(scheme, up, QUIRKS_REFERENCE, fin, to_dev(torch, z[f"rec_{key}_hl"]),
                   to_dev(torch, z[f"rec_{key}_hr"]), out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), z[f"rec_{key}_out"]) < 1e-12


def test_cd6_and_rk3_golden(torch_cuda):
    import nuc3d_b200 as nb
    torch = torch_cuda
    z = golden("operators.npz")
    out = torch.zeros(z["cd6_in"].shape, dtype=torch.float64, device="cuda")
    nb.cd6(float(z["cd6_dx"]), to_dev(torch, z["cd6_in"]), to_dev(torch, z["cd6_hl"]),
           to_dev(torch, z["cd6_hr"]), out)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), z["cd6_out"]) < TOL_OP
    for st in range(3):
        rhs = [to_dev(torch, a) for a in z[f"rk{st}_rhs"]]
        un = [to_dev(torch, a) for a in z[f"rk{st}_un"]]
        ui = [to_dev(torch, a) for a in z[f"rk{st}_ui"]]
        nb.tvdrk3_stage(st, float(z["rk_dt"]), rhs, un, ui)
        torch.cuda.synchronize()
        assert rel_l2(np.stack([u.cpu().numpy() for u in ui]), z[f"rk{st}_out"]) < 1e-15
