"""Deck parsing mirrors the reference's readers (fieldOperator.cpp:100-125,
physicsModel.cpp:66-156, block.cpp:49-61)."""

import pytest

import nuc3d_b200 as nb


def test_decks_round_trip(tmp_path):
    d = nb.BoxDesc(48, 32, 24, lx=6.0, ly=5.0, lz=4.0, scheme=(nb.WENO5Z, nb.CRWENO5, nb.WENO5JS),
                   mach=0.3, reynolds=1234.5, prandtl=0.7, pde_model=nb.EULER3D)
    nb.write_decks(tmp_path, d, {"cfl": 0.4, "endStep": 10})
    r, io, phys = nb.read_decks(tmp_path)
    for k in ("nx", "ny", "nz", "lx", "ly", "lz", "scheme", "mach", "reynolds", "prandtl",
              "pde_model", "gamma", "t_ref", "t_inf"):
        assert getattr(r, k) == getattr(d, k), k
    assert io["cfl"] == 0.4 and io["endStep"] == 10


def test_decks_reject_paths_off_the_gpu_route(tmp_path):
    nb.write_decks(tmp_path, nb.BoxDesc(16, 16, 16))
    p = tmp_path / "inp" / "PhysModel.in"
    p.write_text(p.read_text().replace("RiemannSolver LF", "RiemannSolver Roe"))
    with pytest.raises(ValueError, match="does not exist"):
        nb.read_decks(tmp_path)
    nb.write_decks(tmp_path, nb.BoxDesc(16, 16, 16))
    p.write_text(p.read_text() + "Bogus 1.0\n")
    with pytest.raises(ValueError, match="does not exist"):
        nb.read_decks(tmp_path)


def test_scheme_strings_follow_the_reference(tmp_path):
    """fieldOperator.cpp:128-189: every scheme string the reference registers
    is read, and an unknown string falls back to weno5js."""
    nb.write_decks(tmp_path, nb.BoxDesc(16, 16, 16, scheme=(nb.WENO7JS, nb.WENO5Z, nb.WENO7JS)))
    assert nb.read_decks(tmp_path)[0].scheme == (nb.WENO7JS, nb.WENO5Z, nb.WENO7JS)
    p = tmp_path / "inp" / "Method.in"
    text = p.read_text()
    p.write_text(text.replace("scheme_y_ivs weno5z", "scheme_y_ivs nonesuch"))
    assert nb.read_decks(tmp_path)[0].scheme == (nb.WENO7JS, nb.WENO5JS, nb.WENO7JS)
    for name, sid in (("hccs", nb.HCCS), ("hccs77", nb.HCCS77), ("hccs78", nb.HCCS78),
                      ("weno3js", nb.WENO3JS), ("upwind1st", nb.UPWIND1ST)):
        p.write_text(text.replace("scheme_y_ivs weno5z", f"scheme_y_ivs {name}"))
        assert nb.read_decks(tmp_path)[0].scheme == (nb.WENO7JS, sid, nb.WENO7JS)


@pytest.mark.parametrize("riemann", [0, 1, 2])
def test_riemann_solver_round_trip(tmp_path, riemann):
    """PhysModel.in RiemannSolver LF / AUSM / AUSMp (physicsModel.cpp:16-20)."""
    nb.write_decks(tmp_path, nb.BoxDesc(16, 16, 16, riemann=riemann))
    text = (tmp_path / "inp" / "PhysModel.in").read_text()
    assert f"RiemannSolver {['LF', 'AUSM', 'AUSMp'][riemann]}\n" in text
    assert nb.read_decks(tmp_path)[0].riemann == riemann


def test_differential_scheme_strings_follow_the_reference(tmp_path):
    """fieldOperator.cpp:301-375: scheme_*_vis cd8, cd6 or cd2 per direction;
    an unknown string falls back to cd6."""
    nb.write_decks(tmp_path, nb.BoxDesc(16, 16, 16, vis_scheme=(nb.CD8, nb.CD2, nb.CD6)))
    assert nb.read_decks(tmp_path)[0].vis_scheme == (nb.CD8, nb.CD2, nb.CD6)
    p = tmp_path / "inp" / "Method.in"
    p.write_text(p.read_text().replace("scheme_x_vis cd8", "scheme_x_vis cd4"))
    assert nb.read_decks(tmp_path)[0].vis_scheme == (nb.CD6, nb.CD2, nb.CD6)
