"""Python binding of the nuc3d_b200 C ABI (include/nuc3d_b200.h).

The CUDA path lives in lib/libnuc3d_b200.so (built by build.py).  This module
only marshals arguments: device memory is owned by the caller (torch tensors)
or by a solver context.  There is no CPU fallback — if the library is missing
every entry point raises.
"""

from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field, replace
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parents[2]
LIB_PATH = PKG_ROOT / "lib" / "libnuc3d_b200.so"

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_UNSUPPORTED, ERR_NONFINITE = 0, -1, -2, -3, -4, -5
ERR_TIMEOUT, ERR_CANCELLED = -6, -7
INIT_STATE, INIT_TGV, INIT_HIT = 0, 1, 2
FORCING_NONE, FORCING_CONST, FORCING_BAND = 0, 1, 2
WENO5JS, WENO5Z, CRWENO5, WENO7JS, HCCS, HCCS77, HCCS78, WENO3JS, UPWIND1ST = range(9)
SCHEMES = {"weno5js": WENO5JS, "weno5z": WENO5Z, "crweno5": CRWENO5, "weno7js": WENO7JS,
           "hccs": HCCS, "hccs77": HCCS77, "hccs78": HCCS78, "weno3js": WENO3JS,
           "upwind1st": UPWIND1ST}
TUNING_SLOTS = 27  # NUC3D_TUNING_SLOTS: (scheme id, direction) pairs
PENCIL_DEPTHS = (32, 16, 64)  # the 2.5-D kernels' pencil depths, in tuning order
RIEMANN_LF, RIEMANN_AUSM, RIEMANN_AUSMP = 0, 1, 2
RIEMANNS = {"LF": RIEMANN_LF, "AUSM": RIEMANN_AUSM, "AUSMp": RIEMANN_AUSMP}
CD6, CD2, CD8 = 0, 1, 2  # differential schemes (Method.in scheme_*_vis)
VIS_SCHEMES = {"cd6": CD6, "cd2": CD2, "cd8": CD8}
EULER3D, NAVIERSTOKES3D = 0, 1
SUTHERLAND, CONSTANT, POWERLAW = 0, 1, 2
FP64, MIXED = 0, 1
QUIRK_ZETA_EIGEN = 0x1
QUIRK_WENOZ_BETA2 = 0x2
QUIRK_OFFDIAG_DIV = 0x4
QUIRK_FABS_PRESSURE = 0x8
QUIRK_CRWENO_BOUNDED = 0x10
QUIRKS_REFERENCE = 0x1F
PROF_NAMES = ("prim", "dt", "visc", "inv_x", "inv_y", "inv_z", "update", "residual")
# nuc3d_stats indices (postproc::solveQ averages, turb_para.dat values, dissipation)
STAT_NAMES = ("dudx", "dudy", "dudz", "dvdx", "dvdy", "dvdz", "dwdx", "dwdy", "dwdz",
              "omega_x", "omega_y", "omega_z", "enstrophy", "q_criterion", "helicity", "kinetic",
              "u_rms", "mach_t", "div_rms", "mu_mean", "re_lambda", "taylor_microscale",
              "rho_mean", "eddy_turnover", "skewness", "dissipation")
PROF_CLASSES = len(PROF_NAMES)


class Nuc3dError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"nuc3d error {code}: {msg}")
        self.code = code


class _Desc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
        ("scheme", C.c_int * 3),
        ("pde_model", C.c_int),
        ("visc_model", C.c_int),
        ("gamma", C.c_double), ("mach", C.c_double), ("reynolds", C.c_double),
        ("prandtl", C.c_double), ("t_ref", C.c_double), ("t_inf", C.c_double),
        ("powerlaw_exp", C.c_double),
        ("precision", C.c_int),
        ("quirks", C.c_uint),
        ("forcing", C.c_int),
        ("forcing_amp", C.c_double), ("forcing_hel", C.c_double), ("forcing_k", C.c_double),
        ("riemann", C.c_int),
        ("vis_scheme", C.c_int * 3),
    ]


class _Init(C.Structure):
    _fields_ = [("kind", C.c_int), ("seed", C.c_ulonglong), ("k_peak", C.c_double),
                ("mach_t", C.c_double), ("re_lambda", C.c_double)]


_P5 = C.c_void_p * 5


class _ServeConfig(C.Structure):
    _fields_ = [("precision", C.c_int), ("budget_bytes", C.c_longlong),
                ("max_resident", C.c_int), ("max_chunk_steps", C.c_int),
                ("chunk_ms", C.c_double)]


class _Request(C.Structure):
    _fields_ = [("desc", _Desc), ("nsteps", C.c_int), ("cfl", C.c_double), ("init", _Init),
                ("h_q0", _P5), ("h_q_out", _P5), ("tag", C.c_longlong)]


class _Result(C.Structure):
    _fields_ = [("ticket", C.c_longlong), ("tag", C.c_longlong), ("status", C.c_int),
                ("pad", C.c_int), ("steps", C.c_longlong), ("cells", C.c_longlong),
                ("sim_time", C.c_double), ("dt_last", C.c_double), ("res_last", C.c_double),
                ("reynolds", C.c_double), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double), ("error", C.c_char * 160)]


class _ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong),
                ("failed", C.c_longlong), ("queued", C.c_int), ("resident", C.c_int),
                ("peak_resident", C.c_int), ("pad", C.c_int), ("resident_bytes", C.c_longlong),
                ("peak_resident_bytes", C.c_longlong), ("budget_bytes", C.c_longlong),
                ("batch_steps", C.c_longlong), ("chunks", C.c_longlong),
                ("cell_updates", C.c_longlong), ("launches", C.c_longlong),
                ("graph_captures", C.c_longlong), ("busy_s", C.c_double), ("now_s", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with python nuc3d-cartisian_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        L.nuc3d_last_error.restype = C.c_char_p
        L.nuc3d_version.restype = C.c_char_p
        L.nuc3d_ctx_bytes.restype = C.c_longlong
        L.nuc3d_ctx_bytes.argtypes = [C.POINTER(_Desc)]
        L.nuc3d_ctx_create.argtypes = [C.POINTER(_Desc), C.c_void_p, C.POINTER(C.c_void_p)]
        L.nuc3d_ctx_destroy.argtypes = [C.c_void_p]
        L.nuc3d_set_state_host.argtypes = [C.c_void_p, _P5]
        L.nuc3d_get_state_host.argtypes = [C.c_void_p, _P5]
        L.nuc3d_set_state_host_async.argtypes = [C.c_void_p, _P5]
        L.nuc3d_get_state_host_async.argtypes = [C.c_void_p, _P5]
        L.nuc3d_set_state_device.argtypes = [C.c_void_p, _P5]
        L.nuc3d_get_state_device.argtypes = [C.c_void_p, _P5]
        L.nuc3d_step.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p]
        L.nuc3d_sync.argtypes = [C.c_void_p]
        L.nuc3d_rhs.argtypes = [C.c_void_p, _P5, C.POINTER(C.c_double)]
        L.nuc3d_ctx_time.restype = C.c_double
        L.nuc3d_ctx_time.argtypes = [C.c_void_p]
        L.nuc3d_profile_enable.argtypes = [C.c_void_p, C.c_int]
        L.nuc3d_ctx_copy_lane.argtypes = [C.c_void_p, C.c_int]
        L.nuc3d_profile_read.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.nuc3d_launch_count.restype = C.c_longlong
        L.nuc3d_launch_count.argtypes = [C.c_void_p]
        L.nuc3d_probe_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
        L.nuc3d_batch_create.argtypes = [C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]
        L.nuc3d_batch_destroy.argtypes = [C.c_void_p]
        L.nuc3d_batch_add.argtypes = [C.c_void_p, C.POINTER(_Desc), C.POINTER(C.c_int)]
        for fn in ("remove", "sync"):
            getattr(L, f"nuc3d_batch_{fn}").argtypes = (
                [C.c_void_p, C.c_int] if fn == "remove" else [C.c_void_p])
        L.nuc3d_batch_set_active.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.nuc3d_batch_set_cfl.argtypes = [C.c_void_p, C.c_int, C.c_double]
        for fn in ("set_state_host", "get_state_host", "set_state_device", "get_state_device"):
            getattr(L, f"nuc3d_batch_{fn}").argtypes = [C.c_void_p, C.c_int, _P5]
        L.nuc3d_batch_step.argtypes = [C.c_void_p, C.c_int]
        L.nuc3d_batch_history.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.nuc3d_batch_box_steps.restype = C.c_longlong
        L.nuc3d_batch_box_steps.argtypes = [C.c_void_p, C.c_int]
        L.nuc3d_batch_time.restype = C.c_double
        L.nuc3d_batch_time.argtypes = [C.c_void_p, C.c_int]
        L.nuc3d_batch_profile_enable.argtypes = [C.c_void_p, C.c_int]
        L.nuc3d_batch_profile_read.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.nuc3d_batch_launch_count.restype = C.c_longlong
        L.nuc3d_batch_launch_count.argtypes = [C.c_void_p]
        L.nuc3d_tuning.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.nuc3d_batch_tuning.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.nuc3d_tuning_pencil.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.nuc3d_tuning_tiles.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.nuc3d_batch_tuning_tiles.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.nuc3d_batch_tuning_pencil.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.nuc3d_stats.argtypes = [C.c_void_p, C.c_void_p]
        L.nuc3d_batch_stats.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.nuc3d_spectra.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]
        L.nuc3d_batch_spectra.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int)]
        L.nuc3d_init_state.argtypes = [C.c_void_p, C.POINTER(_Init), C.c_void_p]
        L.nuc3d_batch_init_state.argtypes = [C.c_void_p, C.c_int, C.POINTER(_Init), C.c_void_p]
        L.nuc3d_serve_config_default.argtypes = [C.POINTER(_ServeConfig)]
        L.nuc3d_serve_config_default.restype = None
        L.nuc3d_serve_create.argtypes = [C.POINTER(_ServeConfig), C.POINTER(C.c_void_p)]
        L.nuc3d_serve_destroy.argtypes = [C.c_void_p]
        L.nuc3d_serve_submit.argtypes = [C.c_void_p, C.POINTER(_Request), C.POINTER(C.c_longlong)]
        L.nuc3d_serve_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_double, C.POINTER(_Result)]
        L.nuc3d_serve_info.argtypes = [C.c_void_p, C.POINTER(_ServeStats)]
        L.nuc3d_reconstruct.argtypes = [C.c_int, C.c_int, C.c_uint, C.c_int, C.c_int, C.c_int,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]
        L.nuc3d_cd6.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_void_p]
        L.nuc3d_differential.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]
        L.nuc3d_tvdrk3_stage.argtypes = [C.c_int, C.c_longlong, C.c_double, _P5, _P5, _P5,
                                         C.c_void_p]
        _lib = L
    return _lib


def check(rc: int):
    if rc != OK:
        raise Nuc3dError(rc, lib().nuc3d_last_error().decode())


@dataclass
class BoxDesc:
    """Mirror of nuc3d_box_desc.  Defaults follow the reference decks
    (physicsModel.cpp:23-64, fieldOperator.cpp:22-32) with a 2*pi box."""

    nx: int = 64
    ny: int = 64
    nz: int = 64
    lx: float = 2.0 * math.pi
    ly: float = 2.0 * math.pi
    lz: float = 2.0 * math.pi
    scheme: tuple = (WENO5JS, WENO5JS, WENO5JS)
    pde_model: int = NAVIERSTOKES3D
    visc_model: int = SUTHERLAND
    gamma: float = 1.4
    mach: float = 0.5
    reynolds: float = 1000.0
    prandtl: float = 0.72
    t_ref: float = 110.4
    t_inf: float = 288.0
    powerlaw_exp: float = 0.76
    precision: int = FP64
    quirks: int = QUIRKS_REFERENCE
    forcing: int = FORCING_NONE     # FORCING_CONST: physicsModel::AddForcing_Const; FORCING_BAND
    forcing_amp: float = 0.01       # PhysModel.in Forcing_amplitude
    forcing_hel: float = 0.01       # Forcing_amplitude_hel
    forcing_k: float = 1.0          # Forcing_wave_k
    riemann: int = RIEMANN_LF       # PhysModel.in RiemannSolver: LF, AUSM, AUSMp
    vis_scheme: tuple = (CD6, CD6, CD6)  # Method.in scheme_{x,y,z}_vis: cd6, cd2, cd8

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    def c_struct(self) -> _Desc:
        d = _Desc()
        d.nx, d.ny, d.nz = self.nx, self.ny, self.nz
        d.lx, d.ly, d.lz = self.lx, self.ly, self.lz
        for i in range(3):
            d.scheme[i] = int(self.scheme[i])
        d.pde_model, d.visc_model = int(self.pde_model), int(self.visc_model)
        d.gamma, d.mach, d.reynolds = self.gamma, self.mach, self.reynolds
        d.prandtl, d.t_ref, d.t_inf = self.prandtl, self.t_ref, self.t_inf
        d.powerlaw_exp = self.powerlaw_exp
        d.precision = int(self.precision)
        d.quirks = int(self.quirks)
        d.forcing = int(self.forcing)
        d.forcing_amp, d.forcing_hel, d.forcing_k = self.forcing_amp, self.forcing_hel, self.forcing_k
        d.riemann = int(self.riemann)
        for i in range(3):
            d.vis_scheme[i] = int(self.vis_scheme[i])
        return d

    def device_bytes(self) -> int:
        d = self.c_struct()
        return int(lib().nuc3d_ctx_bytes(C.byref(d)))


def _ptrs5(arrs, n=None, device=None) -> "_P5":
    """Pointers of five contiguous FP64 fields (torch tensors or numpy
    arrays).  The library reads or writes n values through each, so n (when
    given) and the placement (device=True: CUDA tensors, False: host memory)
    are checked here: a short or misplaced buffer is an error, not a copy past
    its end."""
    if len(arrs) != 5:
        raise ValueError(f"need 5 fields, got {len(arrs)}")
    out = _P5()
    for i, a in enumerate(arrs):
        if hasattr(a, "data_ptr"):  # torch tensor
            if not a.is_contiguous() or str(a.dtype) != "torch.float64":
                raise ValueError(f"field {i}: need a contiguous float64 tensor")
            size, on_dev = a.numel(), bool(a.is_cuda)
            out[i] = a.data_ptr()
        else:  # numpy array (host)
            if a.dtype.name != "float64" or not a.flags.c_contiguous:
                raise ValueError(f"field {i}: need a C-contiguous float64 array")
            size, on_dev = a.size, False
            out[i] = a.ctypes.data
        if n is not None and size != n:
            raise ValueError(f"field {i}: {size} values, the box has {n} cells")
        if device is not None and on_dev != device:
            raise ValueError(f"field {i}: expected {'CUDA' if device else 'host'} memory")
    return out


def _on_device(q) -> bool:
    return bool(hasattr(q[0], "is_cuda") and q[0].is_cuda)


def _stream_handle(stream) -> int:
    if stream is None:
        return 0
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    return int(stream)


def _init_struct(init) -> "_Init":
    """init: "tgv", or a dict {"kind": "hit", "seed", "k_peak", "mach_t",
    "re_lambda"} (nuc3d_init_desc)."""
    d = _Init()
    if init == "tgv" or (isinstance(init, dict) and init.get("kind") == "tgv"):
        d.kind = INIT_TGV
        return d
    if not isinstance(init, dict) or init.get("kind") != "hit":
        raise ValueError(f"unknown initial state {init!r}")
    d.kind = INIT_HIT
    d.seed = int(init.get("seed", 0)) & 0xFFFFFFFFFFFFFFFF
    d.k_peak = float(init.get("k_peak", 4.0))
    d.mach_t = float(init.get("mach_t", 0.3))
    d.re_lambda = float(init.get("re_lambda", 0.0) or 0.0)
    return d


def _stats(fn, *args):
    import numpy as np
    out = np.zeros(len(STAT_NAMES))
    check(fn(*args, out.ctypes.data))
    return dict(zip(STAT_NAMES, (float(v) for v in out)))


def _init_info(fn, *args):
    import numpy as np
    info = np.zeros(3)
    check(fn(*args, info.ctypes.data))
    return {"u_rms": float(info[0]), "taylor_microscale": float(info[1]),
            "reynolds": float(info[2])}


class StepPipeline:
    """Advances host-resident states of one box description through `depth`
    solver contexts on their own streams, taking turns: submit() uploads a
    page-locked input state, advances it `nsteps` TVD-RK3 steps and downloads
    the result into a page-locked output, all enqueued without waiting.  The
    contexts' transfers go through the device's copy lanes, so one context's
    upload, another's steps and a third's download run at the same time and
    each transfer has the whole host link.

    A submitted pair of arrays must stay untouched until the same slot is
    submitted again (its previous result has landed when submit() returns)
    or until drain() returns; submit() returns the slot.  A slot's next
    upload and step are enqueued before the wait for its previous result, so
    the wait never holds back work the device could start; drain() also
    checks every context's status (non-finite state, device waits).
    """

    def __init__(self, desc: "BoxDesc", depth: int = 3, cfl: float = 0.5, device=None):
        import torch
        if depth < 1:
            raise ValueError("depth must be >= 1")
        self.desc, self.cfl = desc, cfl
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None else device
        self._streams = [torch.cuda.Stream(dev) for _ in range(depth)]
        self._solvers = []
        try:
            for st in self._streams:
                s = Solver(desc, stream=st)
                s.copy_lane(True)
                self._solvers.append(s)
        except Exception:
            self.close()
            raise
        self._done = [None] * depth  # event after each slot's last download
        self._next = 0

    @property
    def depth(self) -> int:
        return len(self._solvers)

    def warm_up(self, q, nsteps: int = 1):
        """Capture every context's step graph and tune its kernels on state q
        (host arrays), so that submit() only replays."""
        for s in self._solvers:
            s.set_state(q)
            s.step(nsteps, self.cfl, stats=False)
            s.sync()

    def submit(self, q_in, q_out, nsteps: int = 1) -> int:
        import torch
        k = self._next
        self._next = (k + 1) % len(self._solvers)
        s = self._solvers[k]
        s.set_state_async(q_in)
        s.step(nsteps, self.cfl, stats=False)
        if self._done[k] is not None:
            self._done[k].synchronize()  # the slot's previous result has landed
        s.get_state_async(q_out)
        ev = torch.cuda.Event()
        ev.record(self._streams[k])
        self._done[k] = ev
        return k

    def wait(self, slot: int):
        """Blocks until the given slot's last submission has completed and
        checks its context's status."""
        self._solvers[slot].sync()
        self._done[slot] = None

    def drain(self):
        for k in range(len(self._solvers)):
            self.wait(k)

    def close(self):
        for s in self._solvers:
            s.close()
        self._solvers = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Solver:
    """One periodic box resident on the current CUDA device (nuc3d_ctx)."""

    def __init__(self, desc: BoxDesc, stream=None):
        self.desc = desc
        self._cdesc = desc.c_struct()
        h = C.c_void_p()
        check(lib().nuc3d_ctx_create(C.byref(self._cdesc), _stream_handle(stream), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().nuc3d_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> int:
        return self._h.value

    def set_state(self, q):
        """q: 5 host numpy float64 arrays or 5 CUDA float64 tensors."""
        dev = _on_device(q)
        p = _ptrs5(q, self.desc.cells, dev)
        if dev:
            check(lib().nuc3d_set_state_device(self._h, p))
        else:
            check(lib().nuc3d_set_state_host(self._h, p))

    def set_state_async(self, q):
        """Enqueue the upload of 5 page-locked host float64 arrays on the
        solver's stream (nuc3d_set_state_host_async); they must stay valid
        until sync()."""
        check(lib().nuc3d_set_state_host_async(self._h, _ptrs5(q, self.desc.cells, False)))

    def get_state_async(self, out):
        """Enqueue the download into 5 page-locked host float64 arrays
        (nuc3d_get_state_host_async); they hold the state after sync()."""
        check(lib().nuc3d_get_state_host_async(self._h, _ptrs5(out, self.desc.cells, False)))

    def copy_lane(self, on: bool = True):
        """Issue this solver's host transfers in the device's copy lanes
        (nuc3d_ctx_copy_lane): one transfer per direction at a time, in
        submission order, across the solvers whose lane is on."""
        check(lib().nuc3d_ctx_copy_lane(self._h, int(on)))

    def get_state(self, out=None):
        import numpy as np
        if out is None:
            out = [np.zeros(self.desc.shape) for _ in range(5)]
        dev = _on_device(out)
        p = _ptrs5(out, self.desc.cells, dev)
        if dev:
            check(lib().nuc3d_get_state_device(self._h, p))
        else:
            check(lib().nuc3d_get_state_host(self._h, p))
        return out

    def init_state(self, init):
        """Generate the initial state on the device (nuc3d_init_state); a HIT
        init with re_lambda > 0 also sets the Reynolds number (desc is
        updated).  Returns {u_rms, taylor_microscale, reynolds}."""
        d = _init_struct(init)
        info = _init_info(lib().nuc3d_init_state, self._h, C.byref(d))
        self.desc = replace(self.desc, reynolds=info["reynolds"])
        return info

    def stats(self) -> dict:
        """Turbulence statistics of the current state (nuc3d_stats)."""
        return _stats(lib().nuc3d_stats, self._h)

    def spectra(self):
        """The nine shell spectra of the current state (nuc3d_spectra): a
        (9, kmax) array, rows in SPECTRA_NAMES order."""
        return _spectra(lib().nuc3d_spectra, self._h)

    def step(self, nsteps: int, cfl: float, stats: bool = True):
        import numpy as np
        if stats:
            dt = np.zeros(max(nsteps, 1))
            res = np.zeros(max(nsteps, 1))
            check(lib().nuc3d_step(self._h, nsteps, cfl, dt.ctypes.data, res.ctypes.data))
            return dt[:nsteps], res[:nsteps]
        check(lib().nuc3d_step(self._h, nsteps, cfl, None, None))
        return None

    def sync(self):
        check(lib().nuc3d_sync(self._h))

    def rhs(self, out):
        """out: 5 CUDA float64 tensors.  Returns dt_local."""
        dtl = C.c_double(0.0)
        check(lib().nuc3d_rhs(self._h, _ptrs5(out, self.desc.cells, True), C.byref(dtl)))
        return dtl.value

    def time(self) -> float:
        return lib().nuc3d_ctx_time(self._h)

    def profile(self, on: bool):
        check(lib().nuc3d_profile_enable(self._h, int(on)))

    def profile_read(self, reset: bool = True):
        """{class: (milliseconds, launches)} accumulated while profiling."""
        import numpy as np
        ms = np.zeros(PROF_CLASSES)
        n = np.zeros(PROF_CLASSES, dtype=np.int64)
        check(lib().nuc3d_profile_read(self._h, ms.ctypes.data, n.ctypes.data, int(reset)))
        return {name: (float(ms[i]), int(n[i])) for i, name in enumerate(PROF_NAMES)}

    def launch_count(self) -> int:
        return int(lib().nuc3d_launch_count(self._h))

    def tuning(self):
        return _tuning(lib().nuc3d_tuning, self._h, lib().nuc3d_tuning_pencil,
                       lib().nuc3d_tuning_tiles)


class Batch:
    """Many periodic boxes advanced together (nuc3d_batch): one kernel launch
    per kernel class for all boxes, the step replayed as a CUDA graph."""

    def __init__(self, precision=FP64, stream=None):
        h = C.c_void_p()
        check(lib().nuc3d_batch_create(int(precision), _stream_handle(stream), C.byref(h)))
        self._h = h
        self.precision = precision
        self.descs = {}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().nuc3d_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, desc: BoxDesc) -> int:
        d = replace(desc, precision=self.precision).c_struct()
        bid = C.c_int(-1)
        check(lib().nuc3d_batch_add(self._h, C.byref(d), C.byref(bid)))
        self.descs[bid.value] = replace(desc, precision=self.precision)
        return bid.value

    def remove(self, bid: int):
        check(lib().nuc3d_batch_remove(self._h, bid))
        self.descs.pop(bid, None)

    def set_active(self, bid: int, on: bool):
        check(lib().nuc3d_batch_set_active(self._h, bid, int(on)))

    def set_cfl(self, bid: int, cfl: float):
        check(lib().nuc3d_batch_set_cfl(self._h, bid, cfl))

    def set_state(self, bid: int, q):
        dev = _on_device(q)
        p = _ptrs5(q, self.descs[bid].cells, dev)
        if dev:
            check(lib().nuc3d_batch_set_state_device(self._h, bid, p))
        else:
            check(lib().nuc3d_batch_set_state_host(self._h, bid, p))

    def get_state(self, bid: int, out=None):
        import numpy as np
        if out is None:
            out = [np.zeros(self.descs[bid].shape) for _ in range(5)]
        dev = _on_device(out)
        p = _ptrs5(out, self.descs[bid].cells, dev)
        if dev:
            check(lib().nuc3d_batch_get_state_device(self._h, bid, p))
        else:
            check(lib().nuc3d_batch_get_state_host(self._h, bid, p))
        return out

    def init_state(self, bid: int, init):
        """nuc3d_batch_init_state; see Solver.init_state."""
        d = _init_struct(init)
        info = _init_info(lib().nuc3d_batch_init_state, self._h, bid, C.byref(d))
        self.descs[bid] = replace(self.descs[bid], reynolds=info["reynolds"])
        return info

    def stats(self, bid: int) -> dict:
        """Turbulence statistics of box bid (nuc3d_batch_stats)."""
        return _stats(lib().nuc3d_batch_stats, self._h, bid)

    def spectra(self, bid: int):
        """The nine shell spectra of box bid (nuc3d_batch_spectra)."""
        return _spectra(lib().nuc3d_batch_spectra, self._h, bid)

    def step(self, nsteps: int = 1):
        check(lib().nuc3d_batch_step(self._h, nsteps))

    def history(self, bid: int, n: int):
        import numpy as np
        dt = np.zeros(max(n, 1))
        res = np.zeros(max(n, 1))
        check(lib().nuc3d_batch_history(self._h, bid, n, dt.ctypes.data, res.ctypes.data))
        return dt[:n], res[:n]

    def sync(self):
        check(lib().nuc3d_batch_sync(self._h))

    def box_steps(self, bid: int) -> int:
        return int(lib().nuc3d_batch_box_steps(self._h, bid))

    def time(self, bid: int) -> float:
        return lib().nuc3d_batch_time(self._h, bid)

    def profile(self, on: bool):
        check(lib().nuc3d_batch_profile_enable(self._h, int(on)))

    def profile_read(self, reset: bool = True):
        import numpy as np
        ms = np.zeros(PROF_CLASSES)
        n = np.zeros(PROF_CLASSES, dtype=np.int64)
        check(lib().nuc3d_batch_profile_read(self._h, ms.ctypes.data, n.ctypes.data, int(reset)))
        return {name: (float(ms[i]), int(n[i])) for i, name in enumerate(PROF_NAMES)}

    def launch_count(self) -> int:
        return int(lib().nuc3d_batch_launch_count(self._h))

    def tuning(self):
        return _tuning(lib().nuc3d_batch_tuning, self._h, lib().nuc3d_batch_tuning_pencil,
                       lib().nuc3d_batch_tuning_tiles)


class Server:
    """Request loop over a batch (nuc3d_serve_*): solves are admitted by
    device-memory budget, advanced together in chunks (continuous batching)
    by a worker thread inside the library, and collected with wait()."""

    def __init__(self, precision=MIXED, budget_bytes=0, max_resident=256, max_chunk_steps=64,
                 chunk_ms=20.0):
        cfg = _ServeConfig()
        lib().nuc3d_serve_config_default(C.byref(cfg))
        cfg.precision = int(precision)
        cfg.budget_bytes = int(budget_bytes)
        cfg.max_resident = int(max_resident)
        cfg.max_chunk_steps = int(max_chunk_steps)
        cfg.chunk_ms = float(chunk_ms)
        h = C.c_void_p()
        check(lib().nuc3d_serve_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.precision = precision
        self._pending = {}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().nuc3d_serve_destroy(self._h)
            self._h = C.c_void_p()
            self._pending.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, desc: BoxDesc, nsteps: int, cfl: float = 0.5, q0=None, init=None,
               want_state: bool = False, tag: int = 0) -> int:
        """Queue one solve; q0 (5 host float64 arrays) or init ("tgv" or a
        HIT dict, see Solver.init_state) gives its initial state.  Returns the
        ticket."""
        import numpy as np
        r = _Request()
        r.desc = replace(desc, precision=self.precision).c_struct()
        r.nsteps = int(nsteps)
        r.cfl = float(cfl)
        r.tag = int(tag)
        keep = []
        if q0 is not None:
            q0 = [np.ascontiguousarray(a, dtype=np.float64) for a in q0]
            r.init.kind = INIT_STATE
            r.h_q0 = _ptrs5(q0, desc.cells, False)
            keep.append(q0)
        else:
            r.init = _init_struct(init)
        out = None
        if want_state:
            out = [np.empty(desc.shape) for _ in range(5)]
            r.h_q_out = _ptrs5(out, desc.cells, False)
        t = C.c_longlong(-1)
        check(lib().nuc3d_serve_submit(self._h, C.byref(r), C.byref(t)))
        self._pending[t.value] = (keep, out)
        return t.value

    def wait(self, ticket: int = -1, timeout: float | None = None) -> dict:
        """Collect the result of `ticket` (-1: the next to finish)."""
        res = _Result()
        check(lib().nuc3d_serve_wait(self._h, int(ticket), -1.0 if timeout is None else float(timeout),
                                     C.byref(res)))
        _, out = self._pending.pop(res.ticket, (None, None))
        d = {k: getattr(res, k) for k, _ in _Result._fields_ if k not in ("pad", "error")}
        d["error"] = res.error.decode(errors="replace")
        d["state"] = out if res.status == OK else None
        return d

    def stats(self) -> dict:
        st = _ServeStats()
        check(lib().nuc3d_serve_info(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _ServeStats._fields_ if k != "pad"}


SPECTRA_NAMES = ("kin", "kinc", "kins", "kinl", "kinr", "hel", "ens", "den", "pre")


def _spectra(fn, *args):
    import numpy as np
    kmax = C.c_int(0)
    check(fn(*args, None, C.byref(kmax)))
    out = np.zeros((len(SPECTRA_NAMES), kmax.value))
    check(fn(*args, out.ctypes.data, C.byref(kmax)))
    return out


def _tuning(fn, h, fn_pencil=None, fn_tiles=None):
    """{"<scheme>_<dir>": (chosen "<tile cells>x<run length>", {variant: ms per
    launch}), "pencil_depth": (chosen depth, {depth: ms per viscous-flux +
    update pass})}; the sweep variants are "32x1", "32x2", "32x4", "64x2",
    "64x4" (cells per tile along the sweep x faces per thread)."""
    import numpy as np
    rl = np.zeros(TUNING_SLOTS, dtype=np.int32)
    ms = np.zeros(3 * TUNING_SLOTS)
    check(fn(h, rl.ctypes.data, ms.ctypes.data))
    tc = np.full(TUNING_SLOTS, 32, dtype=np.int32)
    ms64 = np.zeros(2 * TUNING_SLOTS)
    if fn_tiles is not None:
        check(fn_tiles(h, tc.ctypes.data, ms64.ctypes.data))
    out = {}
    for sname, s in SCHEMES.items():
        for d, dname in enumerate("xyz"):
            k = s * 3 + d
            if rl[k]:
                times = {f"32x{L}": round(float(ms[k * 3 + v]), 4) for v, L in enumerate((1, 2, 4))}
                if fn_tiles is not None:
                    times.update({f"64x{L}": round(float(ms64[k * 2 + v]), 4)
                                  for v, L in enumerate((2, 4))})
                out[f"{sname}_{dname}"] = (f"{int(tc[k])}x{int(rl[k])}", times)
    if fn_pencil is not None:
        depth = C.c_int(0)
        pms = np.zeros(3)
        check(fn_pencil(h, C.byref(depth), pms.ctypes.data))
        if depth.value:
            out["pencil_depth"] = (depth.value, {D: round(float(pms[v]), 4)
                                                 for v, D in enumerate(PENCIL_DEPTHS)})
    return out


def probe_peak(precision=FP64) -> float:
    """Measured FMA-pipe TFLOP/s of the current device (nuc3d_probe_peak)."""
    t = C.c_double(0.0)
    check(lib().nuc3d_probe_peak(int(precision), C.byref(t)))
    return t.value


# halo width of each reconstruction scheme (the reference's bufferSize,
# fieldOperator.cpp:128-175)
SCHEME_HALO = {WENO5JS: 3, WENO5Z: 3, CRWENO5: 3, WENO7JS: 4, HCCS: 4, HCCS77: 4, HCCS78: 4,
               WENO3JS: 2, UPWIND1ST: 1}


def _operand(t, shape, name):
    """The operator entry points take raw device pointers: check that each
    tensor is a contiguous FP64 CUDA tensor of exactly the size the kernel
    reads or writes, so that a wrong halo width cannot turn into a read
    outside the buffer."""
    if (not hasattr(t, "data_ptr") or not t.is_cuda or str(t.dtype) != "torch.float64"
            or not t.is_contiguous() or tuple(t.shape) != tuple(shape)):
        raise ValueError(f"{name}: need a contiguous float64 CUDA tensor of shape {tuple(shape)}, "
                         f"got {getattr(t, 'dtype', type(t))} {tuple(getattr(t, 'shape', ()))}")


def reconstruct(scheme, upwind, quirks, d_in, d_hl, d_hr, d_out, stream=None):
    """nuc3d_reconstruct on torch CUDA tensors shaped (nz,ny,nx), (nz,ny,H)x2
    (H: the scheme's halo width, SCHEME_HALO), (nz,ny,nx+1)."""
    nz, ny, nx = d_in.shape
    h = SCHEME_HALO.get(scheme, 3)
    _operand(d_in, (nz, ny, nx), "in")
    _operand(d_hl, (nz, ny, h), "halo_l")
    _operand(d_hr, (nz, ny, h), "halo_r")
    _operand(d_out, (nz, ny, nx + 1), "out")
    check(lib().nuc3d_reconstruct(scheme, upwind, quirks, nx, ny, nz, d_in.data_ptr(),
                                  d_hl.data_ptr(), d_hr.data_ptr(), d_out.data_ptr(),
                                  _stream_handle(stream)))


def cd6(dx, d_in, d_hl, d_hr, d_out, stream=None):
    """nuc3d_cd6: (nz,ny,nx) with halos (nz,ny,3)."""
    nz, ny, nx = d_in.shape
    _operand(d_in, (nz, ny, nx), "in")
    _operand(d_hl, (nz, ny, 3), "halo_l")
    _operand(d_hr, (nz, ny, 3), "halo_r")
    _operand(d_out, (nz, ny, nx), "out")
    check(lib().nuc3d_cd6(nx, ny, nz, dx, d_in.data_ptr(), d_hl.data_ptr(), d_hr.data_ptr(),
                          d_out.data_ptr(), _stream_handle(stream)))


def differential(scheme, tile, dx, d_in, d_hl, d_hr, d_out, stream=None):
    """nuc3d_differential: scheme CD6 / CD2 / CD8 with the reference's
    tilesize; halos (nz, ny, tile)."""
    nz, ny, nx = d_in.shape
    _operand(d_in, (nz, ny, nx), "in")
    _operand(d_hl, (nz, ny, tile), "halo_l")
    _operand(d_hr, (nz, ny, tile), "halo_r")
    _operand(d_out, (nz, ny, nx), "out")
    check(lib().nuc3d_differential(scheme, tile, nx, ny, nz, dx, d_in.data_ptr(),
                                   d_hl.data_ptr(), d_hr.data_ptr(), d_out.data_ptr(),
                                   _stream_handle(stream)))


def tvdrk3_stage(stage, dt, d_rhs, d_un, d_ui, stream=None):
    n = d_rhs[0].numel()
    check(lib().nuc3d_tvdrk3_stage(stage, n, dt, _ptrs5(d_rhs, n, True), _ptrs5(d_un, n, True),
                                   _ptrs5(d_ui, n, True), _stream_handle(stream)))


from .decks import read_decks, write_decks  # noqa: E402
from .initial import taylor_green, hit_field  # noqa: E402
