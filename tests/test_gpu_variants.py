"""The autotuned variants are the same arithmetic: the sweeps' runs of 1, 2
or 4 faces per thread on tiles of 32 or 64 cells, and the 2.5-D stencil
kernels' pencil depths.  These
tests pin that they give identical states, so a box's result does not depend
on which variant the autotuner picked for its batch."""

import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]

SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, "oracle"); sys.path.insert(0, "nuc3d-cartisian_b200/python"); sys.path.insert(0, "tests")
from oracle_ctypes import Box, Oracle, WENO5JS, WENO5Z, WENO7
from helpers import desc_from_box
import nuc3d_b200 as nb
prec = int(sys.argv[2])
out = []
for sch in (WENO5JS, WENO5Z, WENO7):
    box = Box(40, 24, 36, scheme=(sch,) * 3, mach=0.3, reynolds=700.0)
    rng = np.random.default_rng(5)
    q = [np.ascontiguousarray(a * (1 + 0.02 * rng.standard_normal(a.shape))) for a in Oracle().tgv(box)]
    with nb.Solver(desc_from_box(box, prec)) as s:
        s.set_state(q)
        s.step(3, 0.5)
        out.append(np.stack(s.get_state()))
np.save(sys.argv[1], np.stack(out))
"""


@pytest.mark.parametrize("precision", [0, 1])
def test_sweep_variants_agree(tmp_path, precision):
    """Runs of 1, 2, 4 faces on 32-cell tiles and, in FP64, of 2, 4 faces on
    64-cell tiles (the 40 x 24 x 36 box leaves partial 64-cell tiles along x
    and z).  Mixed precision runs 32-cell tiles only: its FP32 staging is
    offset by each line's value at the tile's first cell, so another tile
    length would round differently."""
    res = {}
    variants = [(1, 32), (2, 32), (4, 32)] + ([(2, 64), (4, 64)] if precision == 0 else [])
    for run, tile in variants:
        f = tmp_path / f"r{run}_{tile}.npy"
        env = dict(os.environ, NUC3D_SWEEP_RUN=str(run), NUC3D_SWEEP_TILE=str(tile))
        subprocess.run([sys.executable, "-c", SCRIPT, str(f), str(precision)], cwd=ROOT, env=env,
                       check=True)
        res[(run, tile)] = np.load(f)
    for v in variants[1:]:
        diff = np.abs(res[v] - res[(1, 32)]).max()
        print(f"variant {v} vs (1, 32): max abs diff {diff:.3e}")
        assert np.array_equal(res[v], res[(1, 32)])


PENCIL_SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, "oracle"); sys.path.insert(0, "nuc3d-cartisian_b200/python"); sys.path.insert(0, "tests")
from oracle_ctypes import Box, Oracle, WENO5Z
from helpers import desc_from_box
import nuc3d_b200 as nb
prec = int(sys.argv[2])
# nz = 72: partial last pencils at every depth; two boxes in one batch
boxes = [Box(40, 24, 72, scheme=(WENO5Z,) * 3, mach=0.3, reynolds=700.0),
         Box(32, 40, 20, scheme=(WENO5Z,) * 3, mach=0.5, reynolds=300.0)]
out = []
with nb.Batch(prec) as b:
    ids = []
    for box in boxes:
        rng = np.random.default_rng(7)
        q = [np.ascontiguousarray(a * (1 + 0.02 * rng.standard_normal(a.shape)))
             for a in Oracle().tgv(box)]
        i = b.add(desc_from_box(box, prec))
        b.set_state(i, q)
        ids.append(i)
    b.step(3)
    depth = b.tuning()["pencil_depth"][0]
    for i in ids:
        out.append(np.stack(b.get_state(i)).ravel())
np.save(sys.argv[1], np.concatenate(out))
print(depth)
"""


@pytest.mark.parametrize("precision", [0, 1])
def test_pencil_depths_agree(tmp_path, precision):
    """The 2.5-D stencil kernels' pencil depths (16, 32, 64 planes per tile,
    chosen by the autotuner) compute every cell alike: identical states."""
    res = {}
    for depth in (16, 32, 64):
        f = tmp_path / f"d{depth}.npy"
        env = dict(os.environ, NUC3D_PENCIL_DEPTH=str(depth))
        r = subprocess.run([sys.executable, "-c", PENCIL_SCRIPT, str(f), str(precision)], cwd=ROOT,
                           env=env, check=True, capture_output=True, text=True)
        assert int(r.stdout.split()[-1]) == depth
        res[depth] = np.load(f)
    for depth in (16, 64):
        assert np.array_equal(res[depth], res[32])
