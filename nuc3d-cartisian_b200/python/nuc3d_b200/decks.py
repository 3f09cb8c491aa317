"""The reference's plain-text decks (inp/*.in), read and written.

Formats: Method.in key/value (fieldOperator.cpp:21-125), PhysModel.in six
positional "key value" lines then key/value pairs (physicsModel.cpp:66-156),
block.in positional (block.cpp:49-61), IOController.in key/value
(IOcontroller.cpp:10-60).  Unknown PhysModel keys stop the reference
(physicsModel.cpp:148-152); here they raise ValueError.
"""

from __future__ import annotations

from pathlib import Path

from . import (CONSTANT, EULER3D, FORCING_BAND, FORCING_CONST, FORCING_NONE, NAVIERSTOKES3D, RIEMANNS,
               SCHEMES, SUTHERLAND, VIS_SCHEMES, BoxDesc)

_FORCINGS = {"None": FORCING_NONE, "Const": FORCING_CONST, "Band": FORCING_BAND}

def _scheme(name: str) -> int:
    """fieldOperator3d::setMethodIvs* (fieldOperator.cpp:128-189): every
    scheme string the reference registers is on this path; unknown strings
    fall back to weno5js, as the reference's do."""
    return SCHEMES.get(name, SCHEMES["weno5js"])


def _vis_scheme(name: str) -> int:
    """fieldOperator3d::setDiffMethod* (fieldOperator.cpp:301-375): cd8, cd6
    or cd2; unknown strings fall back to cd6, as the reference's do."""
    return VIS_SCHEMES.get(name, VIS_SCHEMES["cd6"])


_METHOD_DEFAULTS = {"scheme_time": "RK3", "scheme_x_ivs": "weno5js", "scheme_y_ivs": "weno5js",
                    "scheme_z_ivs": "weno5js", "scheme_x_vis": "cd6", "scheme_y_vis": "cd6",
                    "scheme_z_vis": "cd6"}
_PHYS_DEFAULTS = {"Reynolds": 1000.0, "Mach": 0.5, "Pt": 0.72, "Rossby": 0.0, "x_center": 3.1415926,
                  "y_center": 3.1415926, "z_center": 0.0, "well_rad": 1.0, "Gamma": 1.4,
                  "T_ref": 110.4, "T_inf": 288.0, "T_wall": 1.0, "Forcing_amplitude": 0.01,
                  "Forcing_amplitude_hel": 0.01, "Forcing_wave_k": 1.0, "Mach_t": 0.3,
                  "k_peak": 8.0}
_IO_DEFAULTS = {"startStep": 0, "endStep": 100000, "postStep": 1, "saveStep": 1000,
                "postSaveStep": 100, "Benchmark": 0, "cfl": 0.5, "tl": 0.0, "dt": 0.01,
                "Binary": "yes", "Tecplot": "yes", "PostProc": "yes"}


def _pairs(text):
    toks = text.split()
    return [(toks[i], toks[i + 1]) for i in range(0, len(toks) - 1, 2)]


def read_decks(dirpath):
    """Return (BoxDesc, io dict, phys dict) for a directory holding inp/."""
    inp = Path(dirpath) / "inp"
    method = dict(_METHOD_DEFAULTS)
    for k, v in _pairs((inp / "Method.in").read_text()):
        if k in method:
            method[k] = v
    toks = (inp / "PhysModel.in").read_text().split()
    if len(toks) < 12:
        raise ValueError("PhysModel.in needs its six positional lines")
    pos = [toks[2 * i + 1] for i in range(6)]  # Neqs EosName RiemannSolver PDEModel ViscousModel Forcing
    if pos[2] not in RIEMANNS:
        # physicsModel.cpp:88-93 prints a warning and then computes no split
        # at all (solveRiemann finds no such name); refuse instead
        raise ValueError(f"Riemann Solver name {pos[2]} does not exist (LF, AUSM, AUSMp)")
    # "Band" (band-limited forcing at a fixed injection rate Forcing_amplitude
    # over 0 < |k| <= Forcing_wave_k) is this library's own keyword; the
    # reference knows None, Const, ABC and TG
    if pos[5] not in _FORCINGS:
        raise ValueError(f"Forcing {pos[5]}: only None, Const and Band are on the B200 path")
    phys = dict(_PHYS_DEFAULTS)
    for k, v in _pairs(" ".join(toks[12:])):
        if k in ("Coriolis", "Centrifugal"):
            if v != "no":
                raise ValueError(f"{k} source is not on the B200 path")
            continue
        if k not in phys:
            raise ValueError(f"word {k} does not exist")
        phys[k] = float(v)
    blk = (inp / "block.in").read_text().split()
    npx, npy, npz = (int(t) for t in blk[0:3])
    if (npx, npy, npz) != (1, 1, 1):
        raise ValueError("the B200 path runs one box per GPU (process topology 1 1 1)")
    nx, ny, nz = (int(t) for t in blk[3:6])
    lx, ly, lz = (float(t) for t in blk[6:9])
    io = dict(_IO_DEFAULTS)
    iof = inp / "IOController.in"
    if iof.exists():
        for k, v in _pairs(iof.read_text()):
            if k in io:
                io[k] = type(_IO_DEFAULTS[k])(float(v)) if not isinstance(_IO_DEFAULTS[k], str) else v
    models = {"Euler3d": EULER3D, "NavierStokes3d": NAVIERSTOKES3D}
    if pos[3] not in models:
        raise ValueError(f"Model Name:{pos[3]} does not exist!")
    visc = {"Sutherland": SUTHERLAND, "Constant": CONSTANT}.get(pos[4], SUTHERLAND)
    desc = BoxDesc(nx=nx, ny=ny, nz=nz, lx=lx, ly=ly, lz=lz,
                   scheme=tuple(_scheme(method[f"scheme_{a}_ivs"]) for a in "xyz"),
                   pde_model=models[pos[3]], visc_model=visc, gamma=phys["Gamma"],
                   mach=phys["Mach"], reynolds=phys["Reynolds"], prandtl=phys["Pt"],
                   t_ref=phys["T_ref"], t_inf=phys["T_inf"],
                   forcing=_FORCINGS[pos[5]],
                   forcing_amp=phys["Forcing_amplitude"], forcing_hel=phys["Forcing_amplitude_hel"],
                   forcing_k=phys["Forcing_wave_k"], riemann=RIEMANNS[pos[2]],
                   vis_scheme=tuple(_vis_scheme(method[f"scheme_{a}_vis"]) for a in "xyz"))
    return desc, io, phys


def write_decks(dirpath, desc, io=None):
    inv = {v: k for k, v in SCHEMES.items()}
    vinv = {v: k for k, v in VIS_SCHEMES.items()}
    inp = Path(dirpath) / "inp"
    inp.mkdir(parents=True, exist_ok=True)
    (inp / "Method.in").write_text(
        "scheme_time RK3\n" + "".join(f"scheme_{a}_ivs {inv[s]}\n" for a, s in zip("xyz", desc.scheme))
        + "".join(f"scheme_{a}_vis {vinv[v]}\n" for a, v in zip("xyz", desc.vis_scheme)))
    model = "NavierStokes3d" if desc.pde_model == NAVIERSTOKES3D else "Euler3d"
    visc = "Constant" if desc.visc_model == CONSTANT else "Sutherland"
    forcing = {v: k for k, v in _FORCINGS.items()}[desc.forcing]
    rname = {v: k for k, v in RIEMANNS.items()}[desc.riemann]
    (inp / "PhysModel.in").write_text(
        f"Neqs 5\nEosName IdealGas\nRiemannSolver {rname}\nPDEModel {model}\nViscousModel {visc}\n"
        f"Forcing {forcing}\nReynolds {desc.reynolds!r}\nMach {desc.mach!r}\nPt {desc.prandtl!r}\n"
        f"Gamma {desc.gamma!r}\nT_ref {desc.t_ref!r}\nT_inf {desc.t_inf!r}\n"
        f"Forcing_amplitude {desc.forcing_amp!r}\nForcing_amplitude_hel {desc.forcing_hel!r}\n"
        f"Forcing_wave_k {desc.forcing_k!r}\n")
    (inp / "block.in").write_text(
        f"1 1 1\n{desc.nx} {desc.ny} {desc.nz}\n{desc.lx!r} {desc.ly!r} {desc.lz!r}\n0.0 0.0 0.0\n")
    io = dict(_IO_DEFAULTS, **(io or {}))
    (inp / "IOController.in").write_text("".join(f"{k} {v}\n" for k, v in io.items()))
