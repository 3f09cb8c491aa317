"""ctypes access to the two CPU checkers.  TEST INFRASTRUCTURE ONLY.

* ``Oracle`` wraps oracle/_build/libnuc3d_oracle.so, the C restatement of the
  reference's RHS + TVD-RK3 path (oracle/nuc3d_oracle.c).
* ``Reference`` wraps oracle/_ref/libnuc3d_ref.so, the reference's own
  translation units compiled where they lie (``make -C oracle ref``).  It only
  exists where the reference sources were present at build time.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, and only as the checker.  Arrays are FP64, x-fastest, shaped
(nz, ny, nx) in numpy (C order), i.e. idx = i + nx*(j + ny*k).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libnuc3d_oracle.so"
REF_SO = HERE / "_ref" / "libnuc3d_ref.so"

WENO5JS, WENO5Z, CRWENO5, WENO7, HCCS, HCCS77, HCCS78, WENO3JS, UPWIND1 = range(9)
SCHEME_NAMES = {WENO5JS: "weno5js", WENO5Z: "weno5z", CRWENO5: "crweno5", WENO7: "weno7js",
                HCCS: "hccs", HCCS77: "hccs77", HCCS78: "hccs78", WENO3JS: "weno3js",
                UPWIND1: "upwind1st"}
SUTHERLAND, CONSTANT, POWERLAW = 0, 1, 2
CD6, CD2, CD8 = 0, 1, 2
VIS_NAMES = {CD6: "cd6", CD2: "cd2", CD8: "cd8"}
# the reference's bufferSize of each inviscid scheme (fieldOperator.cpp:128-290):
# the tilesize its differential schemes get
SCHEME_HALO = {WENO5JS: 3, WENO5Z: 3, CRWENO5: 3, WENO7: 4, HCCS: 4, HCCS77: 4, HCCS78: 4,
               WENO3JS: 2, UPWIND1: 1}
LF, AUSM, AUSMP = 0, 1, 2
RIEMANN_NAMES = {LF: "LF", AUSM: "AUSM", AUSMP: "AUSMp"}
VISC_NAMES = {SUTHERLAND: "Sutherland", CONSTANT: "Constant"}

Q_ZETA_EIGEN = 1 << 0
Q_WENOZ_BETA2 = 1 << 1
Q_OFFDIAG_DIV = 1 << 2
Q_FABS_PRESSURE = 1 << 3
Q_CRWENO_BOUNDED = 1 << 4
QUIRKS_REFERENCE = 0x1F

_DP = C.POINTER(C.c_double)


class _Box(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("scheme", C.c_int * 3),
        ("navier_stokes", C.c_int),
        ("visc_model", C.c_int),
        ("gamma", C.c_double), ("mach", C.c_double), ("reynolds", C.c_double),
        ("prandtl", C.c_double), ("t_ref", C.c_double), ("t_inf", C.c_double),
        ("powerlaw_exp", C.c_double),
        ("quirks", C.c_uint),
        ("riemann", C.c_int),
        ("vis", C.c_int * 3),
    ]


@dataclass
class Box:
    """Box and model parameters; defaults are the Taylor-Green case of the
    reference decks (Re 1600, M 0.1, Pr 0.71, Sutherland, WENO5-JS + CD6)."""

    nx: int
    ny: int
    nz: int
    lx: float = 2.0 * np.pi
    ly: float = 2.0 * np.pi
    lz: float = 2.0 * np.pi
    scheme: tuple = (WENO5JS, WENO5JS, WENO5JS)
    navier_stokes: bool = True
    visc_model: int = SUTHERLAND
    gamma: float = 1.4
    mach: float = 0.1
    reynolds: float = 1600.0
    prandtl: float = 0.71
    t_ref: float = 110.4
    t_inf: float = 288.0
    powerlaw_exp: float = 0.76
    quirks: int = QUIRKS_REFERENCE
    riemann: int = LF
    # Method.in scheme_{x,y,z}_vis (fieldOperator.cpp:301-375)
    vis: tuple = (CD6, CD6, CD6)
    # PhysModel.in Forcing (physicsModel.cpp:50-56): 0 None, 1 Const.  Only
    # the compiled reference runs it (the C restatement has no forcing; its
    # numpy restatement is forcing_oracle.py).
    forcing: int = 0
    forcing_amp: float = 0.01
    forcing_hel: float = 0.01
    forcing_k: float = 1.0

    @property
    def dx(self):
        return self.lx / self.nx  # block.cpp:62-64

    @property
    def dy(self):
        return self.ly / self.ny

    @property
    def dz(self):
        return self.lz / self.nz

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    def c_struct(self) -> _Box:
        b = _Box()
        b.nx, b.ny, b.nz = self.nx, self.ny, self.nz
        b.dx, b.dy, b.dz = self.dx, self.dy, self.dz
        for d in range(3):
            b.scheme[d] = int(self.scheme[d])
        b.navier_stokes = int(self.navier_stokes)
        b.visc_model = int(self.visc_model)
        b.gamma, b.mach, b.reynolds = self.gamma, self.mach, self.reynolds
        b.prandtl, b.t_ref, b.t_inf = self.prandtl, self.t_ref, self.t_inf
        b.powerlaw_exp = self.powerlaw_exp
        b.quirks = int(self.quirks)
        b.riemann = int(self.riemann)
        for d in range(3):
            b.vis[d] = int(self.vis[d])
        return b


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def _ptrs(arrs):
    arr_t = _DP * len(arrs)
    return arr_t(*[_ptr(a) for a in arrs])


def build_oracle():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


class Oracle:
    def __init__(self, so: Path = ORACLE_SO):
        if not Path(so).exists():
            build_oracle()
        self.lib = C.CDLL(str(so))
        L = self.lib
        L.or_rhs.restype = C.c_double
        L.or_reconstruct_field.restype = C.c_int
        L.or_cd6_field.restype = C.c_int

    def reconstruct_field(self, scheme, upwind, quirks, fin, hl, hr):
        nz, ny, nx = fin.shape
        out = np.zeros((nz, ny, nx + 1))
        rc = self.lib.or_reconstruct_field(scheme, upwind, C.c_uint(quirks), nx, ny, nz,
                                           _ptr(fin), _ptr(hl), _ptr(hr), _ptr(out))
        assert rc == 0
        return out

    def cd6_field(self, fin, dx, hl, hr):
        nz, ny, nx = fin.shape
        out = np.zeros_like(fin)
        rc = self.lib.or_cd6_field(nx, ny, nz, C.c_double(dx), _ptr(fin), _ptr(hl), _ptr(hr),
                                   _ptr(out))
        assert rc == 0
        return out

    def cd_field(self, scheme, tile, fin, dx, hl, hr):
        """or_cd_field: scheme CD6/CD2/CD8 with the reference's tilesize;
        halos (nz, ny, tile)."""
        nz, ny, nx = fin.shape
        out = np.zeros_like(fin)
        rc = self.lib.or_cd_field(scheme, tile, nx, ny, nz, C.c_double(dx), _ptr(fin), _ptr(hl),
                                  _ptr(hr), _ptr(out))
        assert rc == 0, rc
        return out

    def con2prim(self, box: Box, q):
        prim = [np.zeros(box.shape) for _ in range(8)]
        b = box.c_struct()
        self.lib.or_con2prim(C.byref(b), _ptrs(q), _ptrs(prim))
        return prim

    def split(self, box: Box, q):
        """con2prim + the box's flux splitting, x-fastest: (prim[8], fl[3][5],
        fr[3][5], eig[3])."""
        prim = self.con2prim(box, q)
        fl = [[np.zeros(box.shape) for _ in range(5)] for _ in range(3)]
        fr = [[np.zeros(box.shape) for _ in range(5)] for _ in range(3)]
        arr15 = _DP * 5
        FL = (arr15 * 3)(*[arr15(*[_ptr(a) for a in fl[d]]) for d in range(3)])
        FR = (arr15 * 3)(*[arr15(*[_ptr(a) for a in fr[d]]) for d in range(3)])
        eig = np.zeros(3)
        b = box.c_struct()
        fn = self.lib.or_lf_split if box.riemann == LF else self.lib.or_ausm_split
        fn(C.byref(b), _ptrs(q), _ptrs(prim), FL, FR, _ptr(eig))
        return prim, fl, fr, eig

    def rk3_stage(self, stage, dt, rhs, un, ui):
        n = rhs[0].size
        self.lib.or_rk3_stage(stage, C.c_long(n), C.c_double(dt), _ptrs(rhs), _ptrs(un),
                              _ptrs(ui))

    def rhs(self, box: Box, q):
        if box.forcing:
            raise NotImplementedError("the C restatement has no forcing (forcing_oracle.py)")
        out = [np.zeros(box.shape) for _ in range(5)]
        b = box.c_struct()
        dt_local = self.lib.or_rhs(C.byref(b), _ptrs(q), _ptrs(out))
        return out, dt_local

    def run_steps(self, box: Box, cfl, nsteps, q):
        q = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in q]
        dt = np.zeros(nsteps)
        res = np.zeros(nsteps)
        b = box.c_struct()
        self.lib.or_run_steps(C.byref(b), C.c_double(cfl), nsteps, _ptrs(q), _ptr(dt), _ptr(res))
        return q, dt, res

    def stats(self, box: Box, q):
        """or_stats: postproc::solveQ's averages and turb_para values plus the
        dissipation (26 values, see nuc3d_oracle.h)."""
        out = np.zeros(26)
        b = box.c_struct()
        self.lib.or_stats(C.byref(b), _ptrs([np.ascontiguousarray(a) for a in q]), _ptr(out))
        return out

    def tgv(self, box: Box, origin=(0.0, 0.0, 0.0)):
        q = [np.zeros(box.shape) for _ in range(5)]
        b = box.c_struct()
        self.lib.or_init_tgv(C.byref(b), C.c_double(origin[0]), C.c_double(origin[1]),
                             C.c_double(origin[2]), _ptrs(q))
        return q


def write_decks(dirpath: Path, box: Box, cfl: float = 0.5):
    """Write the reference's inp/ decks for ``box`` (formats: fieldOperator.cpp:
    100-125, physicsModel.cpp:66-112; the first six PhysModel lines are
    positional, Forcing included)."""
    inp = Path(dirpath) / "inp"
    inp.mkdir(parents=True, exist_ok=True)
    names = [SCHEME_NAMES[s] for s in box.scheme]
    (inp / "Method.in").write_text(
        "scheme_time RK3\n"
        f"scheme_x_ivs {names[0]}\nscheme_y_ivs {names[1]}\nscheme_z_ivs {names[2]}\n"
        f"scheme_x_vis {VIS_NAMES[box.vis[0]]}\nscheme_y_vis {VIS_NAMES[box.vis[1]]}\n"
        f"scheme_z_vis {VIS_NAMES[box.vis[2]]}\n")
    model = "NavierStokes3d" if box.navier_stokes else "Euler3d"
    (inp / "PhysModel.in").write_text(
        f"Neqs 5\nEosName IdealGas\nRiemannSolver {RIEMANN_NAMES[box.riemann]}\n"
        f"PDEModel {model}\nViscousModel {VISC_NAMES[box.visc_model]}\n"
        f"Forcing {'Const' if box.forcing else 'None'}\n"
        f"Reynolds {box.reynolds!r}\nMach {box.mach!r}\nPt {box.prandtl!r}\n"
        f"Gamma {box.gamma!r}\nT_ref {box.t_ref!r}\nT_inf {box.t_inf!r}\n"
        f"Forcing_amplitude {box.forcing_amp!r}\nForcing_amplitude_hel {box.forcing_hel!r}\n"
        f"Forcing_wave_k {box.forcing_k!r}\n")
    # postproc.cpp:35-58: no averaging, simultaneous Q statistics, no files
    (inp / "PostProc.in").write_text(
        "AverageType 0\nAverageStartStep 0\nSimutaneousData 1\nAveragedSaveType 0\n"
        "SimutaneousSaveType 0\nFFTPost 0\n")


class Reference:
    """The reference's own code, driven through oracle/ref/ref_harness.cpp."""

    def __init__(self, so: Path = REF_SO):
        if not Path(so).exists():
            raise FileNotFoundError(f"{so} not built (make -C oracle ref needs the reference)")
        self.lib = C.CDLL(str(so))

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def reconstruct_field(self, scheme, upwind, fin, hl, hr):
        nz, ny, nx = fin.shape
        out = np.zeros((nz, ny, nx + 1))
        rc = self.lib.ref_reconstruct(scheme, upwind, nx, ny, nz, _ptr(fin), _ptr(hl), _ptr(hr),
                                      _ptr(out))
        assert rc == 0
        return out

    def cd6_field(self, fin, dx, hl, hr):
        nz, ny, nx = fin.shape
        out = np.zeros_like(fin)
        self.lib.ref_cd6(nx, ny, nz, C.c_double(dx), _ptr(fin), _ptr(hl), _ptr(hr), _ptr(out))
        return out

    def cd_field(self, scheme, tile, fin, dx, hl, hr):
        nz, ny, nx = fin.shape
        out = np.zeros_like(fin)
        rc = self.lib.ref_cd(scheme, tile, nx, ny, nz, C.c_double(dx), _ptr(fin), _ptr(hl),
                             _ptr(hr), _ptr(out))
        assert rc == 0, rc
        return out

    def rk3_stage(self, stage, dt, rhs, un, ui):
        n = rhs[0].size
        self.lib.ref_rk3_stage(stage, n, C.c_double(dt), _ptrs(rhs), _ptrs(un), _ptrs(ui))

    def split(self, box: Box, q):
        with tempfile.TemporaryDirectory() as td:
            write_decks(Path(td), box)
            prim = [np.zeros(box.shape) for _ in range(8)]
            # rotated layouts: eta (nx, nz, ny) as (slow..fast), zeta (ny, nx, nz)
            shp = [box.shape, (box.nx, box.nz, box.ny), (box.ny, box.nx, box.nz)]
            fl = [np.zeros(shp[d // 5]) for d in range(15)]
            fr = [np.zeros(shp[d // 5]) for d in range(15)]
            eig = np.zeros(3)
            self.lib.ref_split(str(td).encode(), box.nx, box.ny, box.nz, _ptrs(q), _ptrs(prim),
                               _ptrs(fl), _ptrs(fr), _ptr(eig))
        return prim, fl, fr, eig

    def rhs(self, box: Box, q):
        with tempfile.TemporaryDirectory() as td:
            write_decks(Path(td), box)
            out = [np.zeros(box.shape) for _ in range(5)]
            dtl = C.c_double(0.0)
            self.lib.ref_rhs(str(td).encode(), box.nx, box.ny, box.nz, C.c_double(box.dx),
                             C.c_double(box.dy), C.c_double(box.dz), _ptrs(q), _ptrs(out),
                             C.byref(dtl))
        return out, dtl.value

    def stats(self, box: Box, q):
        """postproc::solveQ of the reference (25 values: the 16 averages of
        enstrophy.dat and the 9 turb_para.dat values, printed with 12
        significant digits)."""
        out = np.zeros(25)
        with tempfile.TemporaryDirectory() as td:
            write_decks(Path(td), box)
            rc = self.lib.ref_stats(str(td).encode(), box.nx, box.ny, box.nz, C.c_double(box.dx),
                                    C.c_double(box.dy), C.c_double(box.dz),
                                    _ptrs([np.ascontiguousarray(a) for a in q]), _ptr(out))
        assert rc == 0, rc
        return out

    def spectra(self, box: Box, q):
        """postproc::solveFFT's nine shell spectra, shaped (9, kmax) in the
        order kin, kinc, kins, kinl, kinr, hel, ens, den, pre (12 significant
        digits, as the reference writes them)."""
        kmax = min(box.nx, box.ny, box.nz) // 2
        out = np.zeros((9, kmax))
        with tempfile.TemporaryDirectory() as td:
            write_decks(Path(td), box)
            rc = self.lib.ref_spectra(str(td).encode(), box.nx, box.ny, box.nz,
                                      C.c_double(box.dx), C.c_double(box.dy), C.c_double(box.dz),
                                      _ptrs([np.ascontiguousarray(a) for a in q]), _ptr(out))
        assert rc == 0, rc
        return out

    def run_steps(self, box: Box, cfl, nsteps, q):
        q = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in q]
        dt = np.zeros(nsteps)
        res = np.zeros(nsteps)
        with tempfile.TemporaryDirectory() as td:
            write_decks(Path(td), box, cfl)
            self.lib.ref_run_steps(str(td).encode(), box.nx, box.ny, box.nz, C.c_double(box.dx),
                                   C.c_double(box.dy), C.c_double(box.dz), C.c_double(cfl),
                                   nsteps, _ptrs(q), _ptr(dt), _ptr(res))
        return q, dt, res
