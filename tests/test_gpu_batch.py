"""Batched solver (nuc3d_batch_*): boxes of different sizes, schemes, models
and CFL numbers advanced together must give exactly the same states as each
box advanced alone (no arithmetic crosses boxes; reductions are per box), and
agree with the CPU oracle."""

import numpy as np
import pytest

from helpers import desc_from_box, max_rel_l2
from oracle_ctypes import (CD2, CD6, CD8, CRWENO5, QUIRKS_REFERENCE, Q_CRWENO_BOUNDED, WENO5JS,
                           WENO5Z, Box, Oracle)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def mix_of_boxes():
    rng = np.random.default_rng(8)
    boxes = [
        Box(16, 12, 10, scheme=(WENO5JS,) * 3, mach=0.1, reynolds=1600.0),
        Box(24, 24, 24, scheme=(WENO5Z,) * 3, navier_stokes=False, mach=0.3),
        Box(20, 16, 12, scheme=(CRWENO5,) * 3, mach=0.2, reynolds=600.0),
        Box(32, 18, 9, scheme=(WENO5Z, WENO5JS, CRWENO5), mach=0.25, reynolds=900.0,
            quirks=QUIRKS_REFERENCE & ~Q_CRWENO_BOUNDED),
        Box(12, 20, 16, scheme=(WENO5JS,) * 3, mach=0.15, reynolds=300.0, visc_model=1),
        # cd8 / cd2 / cd6 viscous stencils: the 2.5-D kernels' reach-4 class
        Box(16, 16, 12, scheme=(WENO5Z,) * 3, vis=(CD8, CD2, CD6), mach=0.2, reynolds=500.0),
    ]
    O = Oracle()
    states = [[a * (1 + 0.02 * rng.standard_normal(a.shape)) for a in O.tgv(b)] for b in boxes]
    cfls = [0.5, 0.4, 0.45, 0.3, 0.5, 0.45]
    return boxes, states, cfls


def run_alone(box, q, cfl, nsteps, precision=0):
    import nuc3d_b200 as nb
    with nb.Solver(desc_from_box(box, precision)) as s:
        s.set_state([np.ascontiguousarray(a) for a in q])
        dt, _ = s.step(nsteps, cfl)
        return s.get_state(), dt


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_each_box_alone(torch, precision):
    import nuc3d_b200 as nb
    boxes, states, cfls = mix_of_boxes()
    nsteps = 4
    with nb.Batch(precision) as B:
        ids = [B.add(desc_from_box(b, precision)) for b in boxes]
        for i, q, c in zip(ids, states, cfls):
            B.set_state(i, [np.ascontiguousarray(a) for a in q])
            B.set_cfl(i, c)
        B.step(nsteps)
        B.sync()
        got = [B.get_state(i) for i in ids]
        dts = [B.history(i, nsteps)[0] for i in ids]
    for b, q, c, g, dt in zip(boxes, states, cfls, got, dts):
        ref, dref = run_alone(b, q, c, nsteps, precision)
        for x, y in zip(g, ref):
            np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(dt, dref)


def test_batch_matches_oracle(torch):
    import nuc3d_b200 as nb
    boxes, states, cfls = mix_of_boxes()
    O = Oracle()
    with nb.Batch(0) as B:
        ids = [B.add(desc_from_box(b)) for b in boxes]
        for i, q, c in zip(ids, states, cfls):
            B.set_state(i, [np.ascontiguousarray(a) for a in q])
            B.set_cfl(i, c)
        B.step(2)
        for i, b, q, c in zip(ids, boxes, states, cfls):
            ref, _, _ = O.run_steps(b, c, 2, q)
            assert max_rel_l2(B.get_state(i), ref) < 1e-12


def test_membership_changes_between_steps(torch):
    """Admit a box after 3 steps, retire another, deactivate a third: every
    box's result equals its own history run alone."""
    import nuc3d_b200 as nb
    boxes, states, cfls = mix_of_boxes()
    with nb.Batch(0) as B:
        a = B.add(desc_from_box(boxes[0]))
        b = B.add(desc_from_box(boxes[1]))
        c = B.add(desc_from_box(boxes[2]))
        for i, k in ((a, 0), (b, 1), (c, 2)):
            B.set_state(i, [np.ascontiguousarray(x) for x in states[k]])
            B.set_cfl(i, cfls[k])
        B.step(3)
        d = B.add(desc_from_box(boxes[3]))          # admitted mid-run
        B.set_state(d, [np.ascontiguousarray(x) for x in states[3]])
        B.set_cfl(d, cfls[3])
        frozen = B.get_state(c)
        B.set_active(c, False)                       # paused
        B.step(2)
        B.remove(b)                                  # retired
        B.step(1)
        assert B.box_steps(a) == 6 and B.box_steps(c) == 3 and B.box_steps(d) == 3
        for x, y in zip(B.get_state(c), frozen):
            np.testing.assert_array_equal(x, y)
        ra, _ = run_alone(boxes[0], states[0], cfls[0], 6)
        rd, _ = run_alone(boxes[3], states[3], cfls[3], 3)
        for x, y in zip(B.get_state(a), ra):
            np.testing.assert_array_equal(x, y)
        for x, y in zip(B.get_state(d), rd):
            np.testing.assert_array_equal(x, y)
        B.set_active(c, True)
        B.step(1)
        rc, _ = run_alone(boxes[2], states[2], cfls[2], 4)
        for x, y in zip(B.get_state(c), rc):
            np.testing.assert_array_equal(x, y)


def test_batch_rejects_mismatched_precision(torch):
    import nuc3d_b200 as nb
    with nb.Batch(0) as B:
        d = nb.BoxDesc(16, 16, 16)
        dd = d.c_struct()
        dd.precision = 1
        import ctypes as C
        bid = C.c_int(-1)
        rc = nb.lib().nuc3d_batch_add(B._h, C.byref(dd), C.byref(bid))
        assert rc == nb.ERR_INVALID


def test_status_of_many_boxes_is_checked(torch):
    """nuc3d_batch_sync reads every box's status flags (through mapped host
    memory, up to 32 boxes per export launch): a zero density in box 37 of 40
    (the second export chunk) is reported as a non-finite state, and the same
    batch without it syncs cleanly."""
    import nuc3d_b200 as nb
    box = Box(8, 8, 8, scheme=(WENO5Z,) * 3, mach=0.2, reynolds=400.0)
    q = Oracle().tgv(box)
    for bad in (None, 37):
        with nb.Batch(0) as B:
            ids = [B.add(desc_from_box(box)) for _ in range(40)]
            for i in ids:
                qi = [np.array(a, copy=True) for a in q]
                if i == ids[-3] and bad is not None:
                    qi[0][2, 3, 4] = 0.0  # zero density -> non-finite con2prim
                B.set_state(i, qi)
            B.step(1)
            if bad is None:
                B.sync()
            else:
                with pytest.raises(nb.Nuc3dError) as ei:
                    B.sync()
                assert ei.value.code == nb.ERR_NONFINITE
