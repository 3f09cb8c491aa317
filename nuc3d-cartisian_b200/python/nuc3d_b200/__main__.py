"""Run one seeded decaying-turbulence case on the device and print its
statistics:

    PYTHONPATH=nuc3d-cartisian_b200/python python -m nuc3d_b200 \\
        --n 128 --scheme weno5z --precision mixed --steps 1

The box is (n, n, n) on [0, 2 pi)^3 at Mach 1 with the HIT initial state
generated on the device (k_peak, Mt, Re_lambda as given); the Reynolds
number follows from Re_lambda.  Useful as a small, self-contained workload
for profilers and smoke runs.
"""

from __future__ import annotations

import argparse
import json

from . import FP64, MIXED, RIEMANNS, SCHEMES, BoxDesc, Solver


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m nuc3d_b200")
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--scheme", choices=sorted(SCHEMES), default="weno5z")
    ap.add_argument("--riemann", choices=sorted(RIEMANNS), default="LF")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--cfl", type=float, default=0.5)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--k-peak", type=float, default=4.0)
    ap.add_argument("--mach-t", type=float, default=0.3)
    ap.add_argument("--re-lambda", type=float, default=100.0)
    a = ap.parse_args(argv)
    desc = BoxDesc(a.n, a.n, a.n, mach=1.0, scheme=(SCHEMES[a.scheme],) * 3,
                   riemann=RIEMANNS[a.riemann],
                   precision=MIXED if a.precision == "mixed" else FP64)
    with Solver(desc) as s:
        info = s.init_state({"kind": "hit", "seed": a.seed, "k_peak": a.k_peak,
                             "mach_t": a.mach_t, "re_lambda": a.re_lambda})
        dt, res = s.step(a.steps, a.cfl)
        st = s.stats()
    print(json.dumps({"n": a.n, "scheme": a.scheme, "precision": a.precision, "steps": a.steps,
                      "reynolds": info["reynolds"], "dt_last": float(dt[-1]) if len(dt) else None,
                      "residual_last": float(res[-1]) if len(res) else None,
                      "kinetic": st["kinetic"], "mach_t": st["mach_t"]}))


if __name__ == "__main__":
    main()
