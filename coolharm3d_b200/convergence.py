"""Linear-wave convergence study: the reference's slow magnetosonic mode
(init.linearwave.c, restated in setups.linear_wave) advanced for one wave
period on grids of increasing resolution; after one period the exact
solution is the initial state, so the L1 norm of (final - initial) over the
physical zones is the error, and log2 of the ratio of errors on successive
grids is the convergence order.

    python -m coolharm3d_b200.convergence --sizes 32 64 128 --dims 3

prints one JSON line per precision with the errors and orders.
"""
import json
import math

import numpy as np

from . import PREC_FP64, PREC_MIXED, Engine, setups

VARS = ("rho", "u", "U1", "U2", "U3", "B1", "B2", "B3")


def l1_error(n, dims=3, precision=PREC_FP64, amp=1.0e-4, device=0, max_steps=1_000_000):
    """L1 errors per primitive (mean |final - initial| over the physical
    zones) after one period of the slow mode on an n^dims grid."""
    shape = (n, n, n) if dims == 3 else (n, n, 1)
    prob = setups.linear_wave(shape, amp=amp, precision=precision, device=device)
    e = Engine(prob.desc)
    setups.start(e, prob)
    p0 = e.download()
    t, steps = 0.0, 0
    while t < prob.t_final and steps < max_steps:
        t, _ = e.step(1)
        steps += 1
    p = e.download()
    e.close()
    sl = tuple(slice(3, 3 + x) for x in shape)
    d = np.abs(p[sl] - p0[sl]).reshape(-1, 8).mean(axis=0)
    return {nm: float(d[l]) for l, nm in enumerate(VARS)}, steps, t


def study(sizes=(32, 64, 128), dims=3, precision=PREC_FP64, device=0):
    """Errors on each grid and the order between successive grids."""
    out = {"dims": dims, "precision": "mixed" if precision == PREC_MIXED else "fp64", "sizes": list(sizes),
           "errors": [], "steps": [], "order": []}
    prev = None
    for n in sizes:
        err, steps, t = l1_error(n, dims, precision, device=device)
        out["errors"].append(err)
        out["steps"].append(steps)
        if prev is not None:
            out["order"].append({k: (math.log2(prev[k] / err[k]) if err[k] > 0 and prev[k] > 0 else None)
                                 for k in ("rho", "u", "U1", "U2", "B1", "B2")})
        prev = err
    return out


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--sizes", type=int, nargs="+", default=[32, 64, 128])
    ap.add_argument("--dims", type=int, choices=[2, 3], default=3)
    ap.add_argument("--precision", choices=["fp64", "mixed", "both"], default="both")
    a = ap.parse_args(argv)
    precs = {"fp64": [PREC_FP64], "mixed": [PREC_MIXED], "both": [PREC_FP64, PREC_MIXED]}[a.precision]
    for prec in precs:
        print(json.dumps(study(a.sizes, a.dims, prec)))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
