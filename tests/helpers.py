"""Shared helpers for the test-suite (not product code)."""

from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden(name):
    return np.load(GOLDEN / name)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


def max_rel_l2(A, B):
    return max(rel_l2(a, b) for a, b in zip(A, B))


def box_from_golden(z, scheme, ns):
    from oracle_ctypes import Box
    nz, ny, nx = (int(v) for v in z["shape"])
    return Box(nx, ny, nz, scheme=(scheme,) * 3, navier_stokes=ns, mach=float(z["mach"]),
               reynolds=float(z["reynolds"]), prandtl=float(z["prandtl"]))


def desc_from_box(box, precision=0):
    import nuc3d_b200 as nb
    return nb.BoxDesc(nx=box.nx, ny=box.ny, nz=box.nz, lx=box.lx, ly=box.ly, lz=box.lz,
                      scheme=tuple(box.scheme),
                      pde_model=nb.NAVIERSTOKES3D if box.navier_stokes else nb.EULER3D,
                      visc_model=box.visc_model, gamma=box.gamma, mach=box.mach,
                      reynolds=box.reynolds, prandtl=box.prandtl, t_ref=box.t_ref,
                      t_inf=box.t_inf, powerlaw_exp=box.powerlaw_exp, precision=precision,
                      quirks=box.quirks, riemann=box.riemann, vis_scheme=tuple(box.vis))


def _ulp_perturbed(q, seed):
    rng = np.random.default_rng(seed)
    return [np.nextafter(a, np.where(rng.random(a.shape) < 0.5, -np.inf, np.inf)) for a in q]


def rounding_sensitivity(box, q, nsteps, cfl=0.5, seed=0):
    """How far the oracle's own state after `nsteps` moves when every input
    value is moved by one ulp (max per-field relative L2).  The reference's
    weno7js and hccs are ill-conditioned with respect to rounding (expanded
    Balsara-Shu indicators that cancel terms of size 1e4 f^2, Z weights with
    eps 1e-20 / 1e-40), so two correct implementations that round differently
    agree only to about this level; WENO5 schemes give ~1e-13 here, weno7js
    and hccs ~1e-12 to 1e-9."""
    from oracle_ctypes import Oracle
    O = Oracle()
    a, _, _ = O.run_steps(box, cfl, nsteps, list(q))
    b, _, _ = O.run_steps(box, cfl, nsteps, _ulp_perturbed(q, seed))
    return max_rel_l2(a, b)


def rhs_rounding_sensitivity(box, q, seed=0):
    """The same for one RHS evaluation."""
    from oracle_ctypes import Oracle
    O = Oracle()
    a, _ = O.rhs(box, list(q))
    b, _ = O.rhs(box, _ulp_perturbed(q, seed))
    return max_rel_l2(a, b)
