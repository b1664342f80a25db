"""Linear-wave convergence study.  Two families of waves:

* "reference": the reference's slow magnetosonic mode (init.linearwave.c,
  restated in setups.linear_wave): k = 2 pi (1, 1, 0), B = (1, 0, 0),
  amplitude 1e-4, any N3;
* "fast", "alfven", "slow": one exact RMHD eigenmode of rho 1, p 1,
  B = (1, 1.5, 0), Gamma 4/3 (setups.linear_wave_3d) along the grid diagonal
  k = 2 pi (1, 1, 1) on n^3 grids (k = 2 pi (1, 1, 0) on n^2 x 1 grids),
  amplitude 1e-6.

Each wave is advanced for one period on grids of increasing resolution;
after one period the exact solution is the initial state, so the L1 norm of
(final - initial) over the physical zones is the error, and log2 of the
ratio of errors on successive grids is the convergence order.

    python -m coolharm3d_b200.convergence --mode fast --sizes 32 64 128 256 --dims 3

prints one JSON line per precision with the errors and orders.
"""
import json
import math

import numpy as np

from . import PREC_FP64, PREC_MIXED, RECON_MC, RECON_PPM_MC, Engine, setups

VARS = ("rho", "u", "U1", "U2", "U3", "B1", "B2", "B3")
WAVES = ("reference", "fast", "alfven", "slow")
RECONS = {"ppm_mc": RECON_PPM_MC, "mc": RECON_MC}


def problem(n, dims=3, precision=PREC_FP64, mode="reference", amp=None, recon=RECON_PPM_MC, device=0):
    """The wave of `mode` on an n^dims grid (n^2 x 1 for dims 2); the
    exact modes take the reconstruction `recon`."""
    shape = (n, n, n) if dims == 3 else (n, n, 1)
    if mode == "reference":
        return setups.linear_wave(shape, amp=1.0e-4 if amp is None else amp, precision=precision, device=device)
    kvec = (1, 1, 1) if dims == 3 else (1, 1, 0)
    return setups.linear_wave_3d(shape, mode, amp=1.0e-6 if amp is None else amp, kvec=kvec, recon=recon,
                                 precision=precision, device=device)


def wave_vars(mode, dims=3):
    """The primitives the wave perturbs (the others stay at their
    background value up to roundoff and carry no convergence order)."""
    if mode == "reference":
        return ("rho", "u", "U1", "U2", "B1", "B2")
    dp, _ = setups.eigenmode(mode, 1.0, 1.0, 4.0 / 3.0, (1.0, 1.5, 0.0), (1, 1, 1) if dims == 3 else (1, 1, 0))
    return tuple(v for v, x in zip(VARS, dp) if x != 0.0)


def l1_error(n, dims=3, precision=PREC_FP64, mode="reference", amp=None, recon=RECON_PPM_MC, device=0,
             max_steps=1_000_000):
    """L1 errors per primitive (mean |final - initial| over the physical
    zones) after one period of the wave on an n^dims grid."""
    prob = problem(n, dims, precision, mode, amp, recon, device)
    shape = prob.n
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


def study(sizes=(32, 64, 128), dims=3, precision=PREC_FP64, mode="reference", amp=None, recon=RECON_PPM_MC,
          device=0):
    """Errors on each grid and the order between successive grids."""
    out = {"wave": mode, "dims": dims, "recon": [k for k, v in RECONS.items() if v == recon][0],
           "precision": "mixed" if precision == PREC_MIXED else "fp64", "sizes": list(sizes), "errors": [],
           "steps": [], "order": []}
    names = wave_vars(mode, dims)
    prev = None
    for n in sizes:
        err, steps, t = l1_error(n, dims, precision, mode, amp, recon, device=device)
        out["errors"].append(err)
        out["steps"].append(steps)
        if prev is not None:
            out["order"].append({k: (math.log2(prev[k] / err[k]) if err[k] > 0 and prev[k] > 0 else None)
                                 for k in names})
        prev = err
    return out


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--mode", choices=WAVES, default="reference")
    ap.add_argument("--sizes", type=int, nargs="+", default=[32, 64, 128])
    ap.add_argument("--dims", type=int, choices=[2, 3], default=3)
    ap.add_argument("--amp", type=float, default=None)
    ap.add_argument("--recon", choices=sorted(RECONS), default="ppm_mc", help="reconstruction of the exact modes")
    ap.add_argument("--precision", choices=["fp64", "mixed", "both"], default="both")
    a = ap.parse_args(argv)
    precs = {"fp64": [PREC_FP64], "mixed": [PREC_MIXED], "both": [PREC_FP64, PREC_MIXED]}[a.precision]
    for prec in precs:
        print(json.dumps(study(a.sizes, a.dims, prec, a.mode, a.amp, RECONS[a.recon])), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
