"""The C++ case driver end to end on the GPU: the reference's Taylor-Green
case (decks, device initial state, 10 TVD-RK3 steps, restart file in the
reference's binary layout, block.cpp:609-671) reproduces the reference's own
10-step result, directly and across a restart."""

import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from helpers import golden, max_rel_l2

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "nuc3d-cartisian_b200"))


@pytest.fixture(scope="module")
def driver():
    import build as b
    return b.build_driver()


def tgv_case(tmp, **io):
    import nuc3d_b200 as nb
    d = nb.BoxDesc(24, 24, 24, mach=0.1, reynolds=1600.0, prandtl=0.71)
    nb.write_decks(tmp, d, io=dict({"Benchmark": 2, "cfl": 0.5, "tl": 100.0, "postStep": 0}, **io))
    return d


def read_restart(path, shape):
    raw = np.fromfile(path, dtype=np.float64)
    n = int(np.prod(shape))
    assert raw.size == 1 + 5 * n
    return raw[0], [raw[1 + e * n:1 + (e + 1) * n].reshape(shape) for e in range(5)]


def test_driver_tgv_10_steps_matches_reference(driver, tmp_path):
    d = tgv_case(tmp_path, endStep=10, saveStep=10, postStep=5)
    r = subprocess.run([str(driver), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.count("========step = ") == 10 and "Calculation finished!!" in r.stdout
    z = golden("tgv24_js_10.npz")
    t, q = read_restart(tmp_path / "flowData" / "NUC3d_step_10_ID_0.bin", d.shape)
    assert max_rel_l2(q, z["q10"]) < 1e-12
    assert abs(t - float(np.sum(z["dt"]))) <= 1e-13 * t
    assert len((tmp_path / "enstrophy.dat").read_text().splitlines()) == 2  # steps 5 and 10
    # spectra files as fft::solveShell writes them: "i E_i E_i/sum(E)" per shell
    for name in ("kin", "kinc", "kins", "kinl", "kinr", "hel", "ens", "den", "pre"):
        rows = np.loadtxt(tmp_path / "flowDataTemp" / f"power_shell_10_{name}.dat")
        assert rows.shape == (12, 3) and np.array_equal(rows[:, 0], np.arange(12))
        np.testing.assert_allclose(rows[:, 2], rows[:, 1] / rows[:, 1].sum(), rtol=1e-10)
    kin = np.loadtxt(tmp_path / "flowDataTemp" / "power_shell_10_kin.dat")[:, 1]
    # the Taylor-Green modes (+-1, +-1, +-1) have |k| = sqrt(3): shell 2
    assert kin[0] == 0.0 and kin[2] > 0.5 * kin.sum()


def test_driver_restart_continues_bitwise(driver, tmp_path):
    d = tgv_case(tmp_path, endStep=5, saveStep=5)
    r = subprocess.run([str(driver), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    tgv_case(tmp_path, startStep=5, endStep=10, saveStep=10)
    r = subprocess.run([str(driver), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    z = golden("tgv24_js_10.npz")
    _, q = read_restart(tmp_path / "flowData" / "NUC3d_step_10_ID_0.bin", d.shape)
    assert max_rel_l2(q, z["q10"]) < 1e-12


def test_driver_tecplot_file(driver, tmp_path):
    """IOController "Tecplot yes": block::outputQ_tecplot's ASCII file beside
    the restart file: header, BLOCK-packed mesh vertices, then the
    cell-centred primitives of con2prim, 12 significant digits."""
    d = tgv_case(tmp_path, endStep=2, saveStep=2, Tecplot="yes")
    r = subprocess.run([str(driver), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = (tmp_path / "flowData" / "NUC3d_step_2_id_0.dat").read_text().splitlines()
    assert lines[0] == "title=NUC3d"
    assert lines[1] == "variables=x,y,z,rho,u,v,w,pressure,temperature,e,sound_speed"
    assert lines[2] == " Zone I = 25, J= 25, K=25"
    assert lines[3] == " DATAPACKING=BLOCK, VARLOCATION=([4-11]=CELLCENTERED)"
    vals = np.array([float(v) for v in lines[4:]])
    nv, nc = 25 ** 3, 24 ** 3
    assert vals.size == 3 * nv + 8 * nc
    h = 2.0 * np.pi / 24
    k, j, i = np.meshgrid(np.arange(25), np.arange(25), np.arange(25), indexing="ij")
    for a, idx in enumerate((i, j, k)):
        np.testing.assert_allclose(vals[a * nv:(a + 1) * nv], (h * idx).ravel(), rtol=1e-11, atol=1e-12)
    _, q = read_restart(tmp_path / "flowData" / "NUC3d_step_2_ID_0.bin", d.shape)
    rho, u, v, w = q[0], q[1] / q[0], q[2] / q[0], q[3] / q[0]
    g, m = d.gamma, d.mach
    p = np.abs((q[4] - 0.5 * rho * (u * u + v * v + w * w)) * (g - 1.0))
    want = [rho, u, v, w, p, g * m * m * p / rho, p / rho / (g - 1.0), np.sqrt(g * p / rho)]
    cells = vals[3 * nv:].reshape(8, -1)
    for f in range(8):  # 12 significant digits: within 5e-12 of the value
        np.testing.assert_allclose(cells[f], want[f].ravel(), rtol=1e-11, atol=1e-13)
    # "Tecplot no" writes none
    tgv_case(tmp_path, endStep=2, saveStep=2, Tecplot="no")
    (tmp_path / "flowData" / "NUC3d_step_2_id_0.dat").unlink()
    r = subprocess.run([str(driver), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert not (tmp_path / "flowData" / "NUC3d_step_2_id_0.dat").exists()


def test_case_runner_module(capsys):
    """python -m nuc3d_b200: one seeded HIT case on the device, one JSON line."""
    import json
    from nuc3d_b200.__main__ import main
    main(["--n", "16", "--scheme", "crweno5", "--precision", "mixed", "--steps", "2"])
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert out["steps"] == 2 and out["dt_last"] > 0 and out["kinetic"] > 0


def test_driver_runs_the_differential_schemes_of_its_decks(driver, tmp_path):
    """Method.in scheme_{x,y,z}_vis cd2 / cd6 / cd8 read by the driver and run
    through the C ABI: 5 Taylor-Green steps against the oracle with the same
    schemes (cd8 beside a 3-cell scheme: periodic halos, as on this path)."""
    import nuc3d_b200 as nb
    from oracle_ctypes import CD2, CD6, CD8, WENO5JS, WENO5Z, Box, Oracle
    d = nb.BoxDesc(24, 20, 16, mach=0.2, reynolds=800.0, prandtl=0.71,
                   scheme=(nb.WENO5JS, nb.WENO5Z, nb.WENO5JS),
                   vis_scheme=(nb.CD2, nb.CD6, nb.CD8))
    nb.write_decks(tmp_path, d, io={"Benchmark": 2, "cfl": 0.5, "tl": 100.0, "postStep": 0,
                                    "endStep": 5, "saveStep": 5})
    assert "scheme_z_vis cd8" in (tmp_path / "inp" / "Method.in").read_text()
    r = subprocess.run([str(driver), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    _, q = read_restart(tmp_path / "flowData" / "NUC3d_step_5_ID_0.bin", d.shape)
    box = Box(24, 20, 16, mach=0.2, reynolds=800.0, prandtl=0.71,
              scheme=(WENO5JS, WENO5Z, WENO5JS), vis=(CD2, CD6, CD8))
    O = Oracle()
    q5, _, _ = O.run_steps(box, 0.5, 5, O.tgv(box))
    assert max_rel_l2(q, q5) < 1e-12
