#!/usr/bin/env python3
"""Generate tests/golden/*.npz from the reference's own CPU build.

Run where the reference sources are available (python oracle/build_ref.py
first).  Each fixture holds the state handed to the reference's step_ch()
(after its own init.*.c, or a seeded "stress" state loaded through
oracle/ref_probe.c), the state after `steps` steps (all cells, ghosts
included), pflag, p_gamma, nfail, nfailtot, t, dx[0], M_tot, the run
parameters and the reference's geometry/floor tables.

Stress states draw rho, u from log-uniform ranges down to 1e-6/1e-7,
velocities with 4-vector magnitudes up to ~30 and fields up to ~3, so that
the inversion fallbacks, entropy fix, floors, gamma ceiling and both
interpolation fixups all fire.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import harmtest as ht  # noqa: E402

CASES = [
    # name, config, grid, steps, stress seed (None = reference init)
    ("balsara1_n128_s1", "balsara1", (128, 1, 1), 1, None),
    ("balsara1_n128_s60", "balsara1", (128, 1, 1), 60, None),
    ("balsara1_lf_n64_s20", "balsara1_lf", (64, 1, 1), 20, None),
    ("balsara1_stress_n64_s2", "balsara1", (64, 1, 1), 2, 11),
    ("linwave_12x10x8_s2", "linwave", (12, 10, 8), 2, None),
    ("linwave_stress_10x8x6_s2", "linwave", (10, 8, 6), 2, 7),
    ("linwave_vl_stress_8x8x8_s2", "linwave_vl", (8, 8, 8), 2, 5),
    ("linwave_2d_16x16x1_s3", "linwave", (16, 16, 1), 3, None),
    # no entropy fix: no pow() on the path, the GPU must agree bit for bit
    ("balsara1_noee_stress_n64_s2", "balsara1_noee", (64, 1, 1), 2, 11),
    ("linwave_noee_stress_10x8x6_s2", "linwave_noee", (10, 8, 6), 2, 7),
    ("linwave_noee_stress_12x12x1_s2", "linwave_noee", (12, 12, 1), 2, 17),
    # entropy fix on, one step: pow() differs by ulps between glibc and CUDA
    ("balsara1_stress_n64_s1", "balsara1", (64, 1, 1), 1, 11),
    ("linwave_stress_10x8x6_s1", "linwave", (10, 8, 6), 1, 7),
    # Fishbone-Moncrief torus, Kerr-Schild a=0.9, MKS: the reference's own
    # initial data (loaded back so the counters start at zero), and the same
    # with 5% of the zones replaced by extreme states
    ("torus_24x16x8_s1", "torus", (24, 16, 8), 1, "load"),
    ("torus_24x16x8_s3", "torus", (24, 16, 8), 3, "load"),
    ("torus_stress_16x24x6_s1", "torus", (16, 24, 6), 1, 23),
    # advected field loop, 2D periodic: the reference's own initial data
    ("field_loop_24x24x1_s3", "field_loop", (24, 24, 1), 3, None),
    # whole runs: the reference's own initial data run to its own final time
    # (GridLength[0]): Balsara-1 to t = 0.4, one period of the 2D slow wave;
    # and 200 steps of the small torus
    ("balsara1_n1024_tfinal", "balsara1", (1024, 1, 1), "final", None),
    ("linwave_2d_32x32x1_tfinal", "linwave", (32, 32, 1), "final", None),
    ("torus_24x16x8_s200", "torus", (24, 16, 8), 200, "load"),
    # the torus on the time-dependent metric path (METRIC_GENERAL_DYNAMIC) with
    # the Minkowski-spherical test spacetime: 3D geometry at three time levels,
    # connection by 4th-order differences every substep
    ("torus_dynmink_12x10x6_s1", "torus_dynmink", (12, 10, 6), 1, "load"),
    ("torus_dynmink_12x10x6_s3", "torus_dynmink", (12, 10, 6), 3, "load"),
    # and with the Kerr-Schild test spacetime (static analytic connection)
    ("torus_dynks_12x10x6_s1", "torus_dynks", (12, 10, 6), 1, "load"),
    ("torus_dynks_12x10x6_s3", "torus_dynks", (12, 10, 6), 3, "load"),
    # the circumbinary disk of the post-Newtonian binary setup
    # (init.nz_pn_bbh_disk.c) on the same path, the Minkowski-spherical test
    # spacetime standing in for the PN one the reference does not ship
    ("pnbbh_dynmink_16x12x8_s1", "pnbbh_dynmink", (16, 12, 8), 1, "load"),
    ("pnbbh_dynmink_16x12x8_s3", "pnbbh_dynmink", (16, 12, 8), 3, "load"),
]

# Runs long enough for the flow to amplify a one-ulp change of pow() to O(1):
# besides the reference's result they hold the reference's algorithm run by
# the C oracle (pinned bit for bit to the reference build) with the engine's
# correctly rounded pow() ("cr_*": the result the engine must reproduce) and
# with glibc's pow() moved up one ulp ("ulp_p": the reference's own
# sensitivity to the last bit of pow()).
CHAOTIC = {"torus_24x16x8_s200"}


def oracle_run(lib, out, steps):
    o = ht.Oracle(tuple(int(x) for x in out["n"]), ht.CONFIG_SWITCHES[out["config"]],
                  dict(gam=out["gam"], cour=out["cour"], grid_length=out["grid_length"], startx=out["startx"],
                       dx=out["dx"], geom=out["geom"], conn=out["conn"], cell6=out["cell6_full"],
                       rface=out["rface"], cool_omega=out["cool_omega"], cool_temp=out["cool_temp"]), lib=lib)
    o.set_state(out["p0"], out["t0"], out["dt0"])
    o.step(steps)
    return o.state()


def stress_state(p, seed):
    rng = np.random.default_rng(seed)
    p = p.copy()
    sh = p.shape[:3]
    p[..., 0] = 10 ** rng.uniform(-6, 0, sh)
    p[..., 1] = 10 ** rng.uniform(-7, 0, sh)
    p[..., 2:5] = rng.normal(0, 1.0, sh + (3,)) * 10 ** rng.uniform(-2, 1.5, sh + (1,))
    p[..., 5:8] = rng.normal(0, 1, sh + (3,)) * 10 ** rng.uniform(-2, 0.5, sh + (1,))
    # a direction with one zone holds ghost copies of that zone in the reference
    for a in range(3):
        if sh[a] == 1 + 2 * ht.NG:
            idx = [slice(None)] * 3
            idx[a] = slice(ht.NG, ht.NG + 1)
            p[...] = np.broadcast_to(p[tuple(idx)], p.shape)
    return p


def sprinkle(p, seed):
    """Replace 5% of the zones by extreme states (torus stress fixture)."""
    rng = np.random.default_rng(seed)
    p = p.copy()
    sh = p.shape[:3]
    m = rng.random(sh) < 0.05
    k = int(m.sum())
    p[m, 0] = 10 ** rng.uniform(-8, -1, k)
    p[m, 1] = 10 ** rng.uniform(-9, -1, k)
    p[m, 2:5] = rng.normal(0, 8, (k, 3))
    return p


def make(name, cfg, n, steps, seed):
    r0 = ht.run_ref(cfg, n, 1, dumps=[0], want_geom=True)
    s0 = r0["states"][0]
    geom = r0["geom"]
    if seed is None:
        load = None
        p0, t0, dt0 = s0["p"], s0["t"], s0["dt"]
    elif seed == "load":
        p0, t0, dt0 = s0["p"], s0["t"], s0["dt"]
        load = dict(p=p0, t=t0, dt=dt0)
    elif cfg == "torus":
        p0, t0, dt0 = sprinkle(s0["p"], seed), s0["t"], s0["dt"]
        load = dict(p=p0, t=t0, dt=dt0)
    else:
        p0 = stress_state(s0["p"], seed)
        t0, dt0 = s0["t"], 1e-4
        load = dict(p=p0, t=t0, dt=dt0)
    if steps == "final":
        s, _ = ht.run_ref_final(cfg, n, load=load)
        steps = s["nstep"]
    else:
        r = ht.run_ref(cfg, n, steps, load=load)
        s = r["states"][steps]
    sw = ht.CONFIG_SWITCHES[cfg]
    out = dict(
        config=cfg, n=np.array(n), steps=steps, p0=p0, t0=t0, dt0=dt0,
        p=s["p"], pflag=s["pflag"], gamma=s["gamma"], nfail=s["nfail"], nfailtot=s["nfailtot"],
        t=s["t"], dt=s["dt"], m_tot=s["m_tot"],
        gam=geom["gam"], cour=geom["cour"], grid_length=geom["grid_length"], startx=geom["startx"],
        dx=geom["dx"], geom=geom["geom"], conn=geom["conn"],
        **{"sw_" + k: v for k, v in sw.items()})
    # floors at every cell centre (the engine's builder is checked against these),
    # r and x[RR] along the line (i, N2S, N3S), r at FACE1 and the cooling tables per i
    out["cell_floors"] = geom["cell6"][..., :2]
    out["r_line"] = geom["cell6"][:, ht.NG, ht.NG, 2]
    out["x1_line"] = geom["cell6"][:, ht.NG, ht.NG, 3]
    out["rface"] = geom["rface"]
    out["cool_omega"] = geom["cool_omega"]
    out["cool_temp"] = geom["cool_temp"]
    if name in CHAOTIC:
        out["cell6_full"] = geom["cell6"]
        c = oracle_run(ht.CR_ORACLE, out, steps)
        for k in ("p", "pflag", "gamma", "nfail", "nfailtot", "t", "dt", "m_tot"):
            out["cr_" + k] = c[k]
        out["ulp_p"] = oracle_run("liboracle_powulp.so", out, steps)["p"]
        del out["cell6_full"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "nfailtot", s["nfailtot"].tolist())


if __name__ == "__main__":
    only = sys.argv[1:]
    for c in CASES:
        if not only or c[0] in only:
            make(*c)
