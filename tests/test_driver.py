"""The C++ case driver (nuc3d-cartisian_b200/host/nuc3d_run.cpp) reads the
reference's decks (inp/*.in) exactly as the Python deck reader does, and
answers bad decks with the reference's messages and a non-zero exit (no GPU
needed for either)."""

import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "nuc3d-cartisian_b200"))


@pytest.fixture(scope="module")
def driver():
    import build as b
    if not b.LIB.exists():
        pytest.skip("library not built")
    return b.build_driver()


def run(driver, *args):
    return subprocess.run([str(driver), *map(str, args)], capture_output=True, text=True, timeout=60)


def parsed(text):
    t = text.split()
    return {t[i]: t[i + 1] for i in range(0, len(t) - 1, 2)}


@pytest.mark.parametrize("kw", [
    dict(nx=24, ny=20, nz=16, mach=0.1, reynolds=1600.0, prandtl=0.71),
    dict(nx=40, ny=32, nz=24, scheme=(1, 2, 0), pde_model=0, mach=0.3, reynolds=250.5),
    dict(nx=16, ny=16, nz=16, scheme=(2, 2, 2), visc_model=1, gamma=1.3, lx=1.5, ly=2.5, lz=3.5),
    dict(nx=20, ny=18, nz=16, scheme=(3, 0, 3), riemann=1),
    dict(nx=16, ny=16, nz=16, riemann=2, pde_model=0),
    dict(nx=24, ny=16, nz=12, scheme=(4, 2, 4)),
    dict(nx=32, ny=32, nz=32, forcing=1, forcing_amp=0.02, forcing_hel=0.1, forcing_k=2.0),
    dict(nx=32, ny=32, nz=32, forcing=2, forcing_amp=0.3, forcing_k=2.0),
    dict(nx=20, ny=16, nz=16, scheme=(3, 7, 8), vis_scheme=(2, 1, 0)),
])
def test_driver_reads_decks_like_the_python_reader(driver, tmp_path, kw):
    import nuc3d_b200 as nb
    d = nb.BoxDesc(**kw)
    nb.write_decks(tmp_path, d, io={"cfl": 0.45, "endStep": 7, "tl": 3.5})
    ref, io, _ = nb.read_decks(tmp_path)
    r = run(driver, tmp_path, "--check-decks")
    assert r.returncode == 0, r.stderr
    got = parsed(r.stdout)
    assert [int(got[k]) for k in ("nx", "ny", "nz")] == [ref.nx, ref.ny, ref.nz]
    assert [float(got[k]) for k in ("lx", "ly", "lz")] == [ref.lx, ref.ly, ref.lz]
    assert [int(x) for x in r.stdout.split("scheme ")[1].split()[:3]] == list(ref.scheme)
    assert int(got["pde"]) == ref.pde_model and int(got["visc"]) == ref.visc_model
    for k, v in (("gamma", ref.gamma), ("mach", ref.mach), ("reynolds", ref.reynolds),
                 ("prandtl", ref.prandtl), ("t_ref", ref.t_ref), ("t_inf", ref.t_inf),
                 ("cfl", io["cfl"]), ("tl", io["tl"])):
        assert float(got[k]) == v
    assert float(got["endStep"]) == io["endStep"]
    assert int(got["forcing"]) == ref.forcing
    assert int(got["riemann"]) == ref.riemann
    assert [int(x) for x in r.stdout.split(" vis ")[1].split()[:3]] == list(ref.vis_scheme)
    for k in ("forcing_amp", "forcing_hel", "forcing_k"):
        assert float(got[k]) == getattr(ref, k)


def test_driver_rejects_what_the_path_does_not_cover(driver, tmp_path):
    import nuc3d_b200 as nb
    r = run(driver, tmp_path / "nothing")
    assert r.returncode != 0 and "does not exist" in r.stderr
    nb.write_decks(tmp_path, nb.BoxDesc(16, 16, 16))
    inp = tmp_path / "inp"
    (inp / "block.in").write_text("2 1 1\n16 16 16\n1 1 1\n0 0 0\n")
    r = run(driver, tmp_path, "--check-decks")
    assert r.returncode != 0 and "topology" in r.stderr
    nb.write_decks(tmp_path, nb.BoxDesc(16, 16, 16))
    text = (inp / "PhysModel.in").read_text().replace("Forcing None", "Forcing ABC")
    (inp / "PhysModel.in").write_text(text)
    r = run(driver, tmp_path, "--check-decks")
    assert r.returncode != 0 and "Forcing" in r.stderr
    nb.write_decks(tmp_path, nb.BoxDesc(16, 16, 16))
    (inp / "PhysModel.in").write_text((inp / "PhysModel.in").read_text() + "Bogus 1.0\n")
    r = run(driver, tmp_path, "--check-decks")
    assert r.returncode != 0 and "word Bogus does not exist" in r.stderr
    nb.write_decks(tmp_path, nb.BoxDesc(16, 16, 16))
    text = (inp / "Method.in").read_text().replace("scheme_time RK3", "scheme_time RK4")
    (inp / "Method.in").write_text(text)
    r = run(driver, tmp_path, "--check-decks")
    assert r.returncode != 0 and "RK4" in r.stderr
    r = run(driver, "--help")
    assert r.returncode == 0 and "usage" in r.stdout
