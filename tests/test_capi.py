"""The C-ABI library loads without a GPU and exports every entry point that
include/nuc3d_b200.h declares; argument validation answers with status codes
before any device work (the reference prints and exits instead,
weno5js.cpp:32-34)."""

import ctypes as C
import re
from pathlib import Path

import pytest

import nuc3d_b200 as nb

HEADER = Path(__file__).resolve().parents[1] / "include" / "nuc3d_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"NUC3D_API[^;(]*?\b(nuc3d_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 15
    L = nb.lib()
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_version_and_default_desc():
    assert b"sm_100a" in nb.lib().nuc3d_version()
    d = nb._Desc()
    nb.lib().nuc3d_box_desc_default(C.byref(d))
    # physicsModel.cpp:25-35 defaults, fieldOperator.cpp:22-32 (weno5js, cd6, RK3)
    assert (d.nx, d.ny, d.nz) == (64, 64, 64)
    assert d.reynolds == 1000.0 and d.mach == 0.5 and d.prandtl == 0.72 and d.gamma == 1.4
    assert d.t_ref == 110.4 and d.t_inf == 288.0
    assert list(d.scheme) == [0, 0, 0] and d.quirks == nb.QUIRKS_REFERENCE


def test_ctx_bytes_accounting():
    d = nb.BoxDesc(32, 32, 32)
    fp64 = d.device_bytes()
    mixed = nb.BoxDesc(32, 32, 32, precision=nb.MIXED).device_bytes()
    assert fp64 >= 21 * 32 ** 3 * 8 + 14 * 32 ** 3 * 8
    assert mixed < fp64
    assert nb.BoxDesc(4, 32, 32).device_bytes() == -1  # too small a box


@pytest.mark.parametrize("args,code", [
    ((12, 1, 0, 16, 2, 2), nb.ERR_UNSUPPORTED),  # no such scheme
    ((9, 1, 0, 16, 2, 2), nb.ERR_UNSUPPORTED),   # one past upwind1st
    ((4, 1, 0, 8, 2, 2), nb.ERR_INVALID),        # hccs line too short
    ((5, 1, 0, 8, 2, 2), nb.ERR_INVALID),        # hccs77 line too short
    ((5, 1, 0, 5000, 2, 2), nb.ERR_INVALID),     # hccs77 line too long
    ((3, 1, 0, 5, 2, 2), nb.ERR_INVALID),        # weno7js line too short
    ((0, 2, 0, 16, 2, 2), nb.ERR_INVALID),       # no such direction
    ((0, 1, 0, 5, 2, 2), nb.ERR_INVALID),        # line too short
    ((2, 1, 0, 5000, 2, 2), nb.ERR_INVALID),     # crweno5 line too long
])
def test_reconstruct_validation_without_device(args, code):
    rc = nb.lib().nuc3d_reconstruct(*args, None, None, None, None, None)
    assert rc == code
    assert nb.lib().nuc3d_last_error()


@pytest.mark.parametrize("args,code", [
    ((3, 4, 16, 2, 2, 0.1), nb.ERR_UNSUPPORTED),  # no such differential scheme
    ((2, 3, 16, 2, 2, 0.1), nb.ERR_INVALID),      # cd8 reads 4 cells: tilesize 3 too small
    ((0, 2, 16, 2, 2, 0.1), nb.ERR_INVALID),      # cd6 reads 3 cells
    ((1, 5, 16, 2, 2, 0.1), nb.ERR_INVALID),      # tilesize above 4
    ((1, 2, 3, 2, 2, 0.1), nb.ERR_INVALID),       # line shorter than two tiles
    ((1, 1, 16, 2, 2, 0.0), nb.ERR_INVALID),      # dx must be > 0
])
def test_differential_validation_without_device(args, code):
    rc = nb.lib().nuc3d_differential(*args, None, None, None, None, None)
    assert rc == code
    assert nb.lib().nuc3d_last_error()


def test_operator_wrappers_check_their_operands():
    """The Python operator wrappers refuse tensors the kernels would read
    outside of (wrong halo width, host memory) before calling the library."""
    torch = pytest.importorskip("torch")
    a = torch.zeros((2, 2, 16), dtype=torch.float64)
    h = torch.zeros((2, 2, 4), dtype=torch.float64)
    with pytest.raises(ValueError):
        nb.differential(nb.CD8, 4, 0.1, a, h, h, a.clone())  # host tensors
    with pytest.raises(ValueError):
        nb.reconstruct(nb.WENO5JS, 1, nb.QUIRKS_REFERENCE, a, h, h,
                       torch.zeros((2, 2, 17), dtype=torch.float64))


def test_ctx_create_rejects_bad_descriptions_without_device():
    L = nb.lib()
    h = C.c_void_p()
    for bad in (nb.BoxDesc(4, 16, 16), nb.BoxDesc(16, 16, 16, scheme=(0, 9, 0)),
                nb.BoxDesc(16, 16, 16, mach=-1.0), nb.BoxDesc(16, 16, 16, precision=3),
                nb.BoxDesc(16, 16, 16, riemann=3), nb.BoxDesc(16, 16, 16, vis_scheme=(0, 3, 0))):
        d = bad.c_struct()
        assert L.nuc3d_ctx_create(C.byref(d), None, C.byref(h)) in (nb.ERR_INVALID,
                                                                    nb.ERR_UNSUPPORTED)
        assert not h.value


def _c_layout(struct, fields):
    """sizeof and offsetof of a header struct, from a gcc-compiled probe."""
    import shutil
    import subprocess
    import tempfile
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    lines = [f'printf("%zu\\n", sizeof({struct}));']
    lines += [f'printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    src = ("#include <stddef.h>\n#include <stdio.h>\n#include \"nuc3d_b200.h\"\n"
           "int main(void) {\n" + "\n".join(lines) + "\nreturn 0; }\n")
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "probe.c"
        exe = Path(d) / "probe"
        c.write_text(src)
        subprocess.run(["gcc", "-I", str(HEADER.parent), str(c), "-o", str(exe)], check=True)
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    vals = [int(v) for v in out.split()]
    return vals[0], vals[1:]


@pytest.mark.parametrize("cname,ctype", [
    ("nuc3d_box_desc", "_Desc"), ("nuc3d_init_desc", "_Init"),
    ("nuc3d_serve_config", "_ServeConfig"), ("nuc3d_solve_request", "_Request"),
    ("nuc3d_solve_result", "_Result"), ("nuc3d_serve_stats", "_ServeStats"),
])
def test_binding_structs_match_the_header(cname, ctype):
    ct = getattr(nb, ctype)
    names = [f for f, _ in ct._fields_]
    size, offs = _c_layout(cname, names)
    assert size == C.sizeof(ct)
    assert offs == [getattr(ct, f).offset for f in names]


def test_serve_and_init_validation_without_device():
    L = nb.lib()
    cfg = nb._ServeConfig()
    L.nuc3d_serve_config_default(C.byref(cfg))
    assert cfg.precision == nb.MIXED and cfg.max_resident == 256 and cfg.chunk_ms == 20.0
    cfg.precision = 7
    h = C.c_void_p()
    assert L.nuc3d_serve_create(C.byref(cfg), C.byref(h)) == nb.ERR_UNSUPPORTED
    assert not h.value
    assert L.nuc3d_serve_submit(None, None, None) == nb.ERR_INVALID
    assert L.nuc3d_serve_wait(None, 0, 0.0, None) == nb.ERR_INVALID
    assert L.nuc3d_init_state(None, None, None) == nb.ERR_INVALID
    assert L.nuc3d_serve_destroy(None) == nb.OK


def test_field_pointers_are_size_checked():
    """Five fields of exactly the box's cell count, in the memory the call
    expects; anything else is refused before the library copies."""
    import numpy as np
    good = [np.zeros((4, 4, 8)) for _ in range(5)]
    nb._ptrs5(good, 128, False)
    with pytest.raises(ValueError):
        nb._ptrs5(good, 129, False)          # wrong size
    with pytest.raises(ValueError):
        nb._ptrs5(good[:4], 128, False)      # four fields
    with pytest.raises(ValueError):
        nb._ptrs5(good, 128, True)           # host memory where device memory is expected
    with pytest.raises(ValueError):
        nb._ptrs5([a.astype(np.float32) for a in good], 128, False)
    with pytest.raises(ValueError):
        nb._ptrs5([np.zeros((8, 4, 4)).T for _ in range(5)], 128, False)  # not C-contiguous
