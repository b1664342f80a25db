"""Loading of the golden fixtures of tests/golden (made by make_golden.py)."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# runs long enough that the reference's own last-bit sensitivity is O(1e-4):
# compared in tests/test_t_final.py against the stored correctly rounded run
CHAOTIC = {"torus_24x16x8_s200"}


def _all():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def names():
    """Fixtures of the static metrics (METRIC_DIM 0 and 2), which the C oracle
    restates too."""
    return [n for n in _all() if "_dyn" not in n]


def dynamic_names():
    """Fixtures of the time-dependent metric path (METRIC_DIM 3): compared
    with the engine directly (tests/test_dynamic_metric.py)."""
    return [n for n in _all() if "_dyn" in n]


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    d["config"] = str(d["config"])
    d["n"] = tuple(int(x) for x in d["n"])
    d["steps"] = int(d["steps"])
    d["sw"] = {k[3:]: int(d[k]) for k in z.files if k.startswith("sw_")}
    for k in ("t0", "dt0", "t", "dt", "m_tot", "gam", "cour"):
        d[k] = float(d[k])
    return d


def cell6_of(f):
    """Per-cell (rhoflr, uuflr, r, ...) array with the fields the step reads."""
    shape = tuple(x + 6 for x in f["n"])
    c = np.zeros(shape + (6,))
    c[..., :2] = f["cell_floors"]
    c[:, :, :, 2] = f["r_line"][:, None, None]
    # x[RR] of the line (i, N2S, N3S), which RESCALE_R scales by; the same as
    # r except where a setup left x[RR] changed (fixtures recorded before the
    # column was kept have x[RR] = r)
    c[:, :, :, 3] = f.get("x1_line", f["r_line"])[:, None, None]
    return c


def geomd(f, cell6=None):
    """Descriptor dict for harmtest.Oracle from a fixture."""
    return dict(gam=f["gam"], cour=f["cour"], grid_length=f["grid_length"], startx=f["startx"], dx=f["dx"],
                geom=f["geom"], conn=f["conn"], cell6=cell6 if cell6 is not None else cell6_of(f),
                rface=f["rface"], cool_omega=f["cool_omega"], cool_temp=f["cool_temp"])
