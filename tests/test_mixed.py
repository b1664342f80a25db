"""The mixed-precision form (HG_PREC_MIXED: reconstruction and HLL/LF face
fluxes in FP32, everything else in FP64) against the FP64 engine on the same
inputs.  Tolerances are relative L1 norms per primitive over the physical
zones, sum |mixed - fp64| / sum |fp64|, stated with each test; the corner
divergence of B (divb_calc, diag.c:503-612) must stay at FP64 round-off
because the constrained-transport update stays FP64."""
import numpy as np
import pytest

import coolharm3d_b200 as hg
import fixtures
from coolharm3d_b200 import torus

pytestmark = pytest.mark.gpu

NAMES = ["rho", "u", "U1", "U2", "U3", "B1", "B2", "B3"]


def l1_rel(a, b):
    a, b = a[3:-3, 3:-3, 3:-3], b[3:-3, 3:-3, 3:-3]
    return {nm: float(np.abs(a[..., l] - b[..., l]).sum() / max(np.abs(b[..., l]).sum(), 1e-300))
            for l, nm in enumerate(NAMES)}


def fixture_engine(f, precision):
    sw = f["sw"]
    d = hg.make_desc(f["n"], f["gam"], f["cour"], f["dx"], f["startx"], f["grid_length"], t=f["t0"],
                     recon=sw["recon"], flux=sw["flux"], ct_para=sw["ct_para"], bc=sw["bc"],
                     metric_dim=sw["metric_dim"], use_ee=sw["ee"], cooling=sw["cooling"], rescale_r=sw["rescale"],
                     precision=precision)
    e = hg.Engine(d)
    if sw["metric_dim"] == 0:
        geom, cell6 = hg.minkowski_tables(d)
        e.set_geometry(geom)
        e.set_cell_data(cell6)
    else:
        e.set_geometry(f["geom"], f["conn"])
        e.set_cell_data(fixtures.cell6_of(f), f["rface"] if sw["rescale"] else None)
    if sw["cooling"]:
        e.set_cooling_tables(f["cool_omega"], f["cool_temp"])
    e.upload(f["p0"])
    e.set_time(f["t0"], f["dt0"])
    return e


# (fixture, steps, relative L1 tolerance per primitive)
CASES = [("torus_24x16x8_s3", 3, 1e-5), ("linwave_12x10x8_s2", 2, 1e-6), ("balsara1_n128_s60", 60, 1e-5)]


@pytest.mark.parametrize("name,steps,tol", CASES)
def test_mixed_close_to_fp64(name, steps, tol):
    f = fixtures.load(name)
    e64 = fixture_engine(f, hg.PREC_FP64)
    e32 = fixture_engine(f, hg.PREC_MIXED)
    e64.step(steps)
    e32.step(steps)
    p64, p32 = e64.download(), e32.download()
    assert np.isfinite(p32).all()
    err = l1_rel(p32, p64)
    print(name, {k: "%.2e" % v for k, v in err.items()})
    bad = {k: v for k, v in err.items() if v > tol}
    assert not bad, bad
    assert err != {k: 0.0 for k in NAMES}  # the FP32 path really ran
    e64.close()
    e32.close()


def divb(p, gdet, invdx):
    """|div B| at the corners (i-1/2, j-1/2, k-1/2) whose eight zones are all
    physical, from the zone-centred B^i and sqrt(-g) (divb_calc,
    diag.c:503-612)."""
    gB = [p[..., 5 + a] * gdet[:, :, None] for a in range(3)]
    sl = lambda di, dj, dk: (slice(4 - di, p.shape[0] - 3 - di), slice(4 - dj, p.shape[1] - 3 - dj),
                             slice(4 - dk, p.shape[2] - 3 - dk))
    tot = 0.
    for a in range(3):
        s = 0.
        for di in (0, 1):
            for dj in (0, 1):
                for dk in (0, 1):
                    sign = -1.0 if (di, dj, dk)[a] == 1 else 1.0
                    s = s + sign * gB[a][sl(di, dj, dk)]
        tot = tot + s * invdx[a]
    return 0.25 * np.abs(tot)


@pytest.mark.parametrize("precision", [hg.PREC_FP64, hg.PREC_MIXED])
def test_divb_stays_at_roundoff(precision):
    n = (24, 16, 8)
    d = torus.torus_desc(n, precision=precision)
    t = torus.torus_tables(d)
    e = hg.Engine(d)
    e.set_geometry(t["geom"], t["conn"])
    e.set_cell_data(t["cell6"], t["rface"])
    e.set_cooling_tables(t["cool_omega"], t["cool_temp"])
    p0 = torus.set_torus(e, d, t, seed=5)
    gdet = t["geom"].reshape(5, n[0] + 6, n[1] + 6, 42)[3, :, :, 32]
    invdx = [1.0 / d.dx[a] for a in (1, 2, 3)]
    scale = max(np.abs(p0[..., 5 + a] * gdet[:, :, None]).max() * invdx[a] for a in range(3))
    e.set_time(d.t, d.dx[0])
    e.step(10)
    p = e.download()
    assert np.abs(p[..., 5:8] - p0[..., 5:8]).max() > 0  # the field evolved
    rel = divb(p, gdet, invdx).max() / scale
    print("precision", precision, "max |div B| / scale", rel)
    assert rel < 1e-12
    e.close()


def test_mixed_launch_configurations_agree():
    """The FP32 flux kernels with x1 strips and other strip lengths give the
    per-face FP32 result up to FP32 rounding (the compiler may contract
    multiply-adds differently in each kernel)."""
    f = fixtures.load("torus_24x16x8_s3")
    runs = []
    for x1, nf in ((0, 2), (1, 1), (1, 3)):
        e = fixture_engine(f, hg.PREC_MIXED)
        c = e.launch_config()
        c.strip_x1, c.strip_faces = x1, nf
        e.set_launch_config(c)
        e.step(3)
        runs.append(e.download())
        e.close()
    for p in runs[1:]:
        err = l1_rel(p, runs[0])
        assert max(err.values()) < 1e-5, err


@pytest.mark.parametrize("name", ["torus_stress_16x24x6_s1", "linwave_stress_10x8x6_s2", "balsara1_stress_n64_s1"])
def test_fp32_copy_stays_current(name):
    """The FP32 copy the mixed form's flux kernels read is written by every
    kernel that writes the state and refreshed by every host update, so it
    equals the FP64 state rounded to float after the set-up, after steps
    (fixups and boundaries included), after autotuning and in a batch."""
    f = fixtures.load(name)
    e = fixture_engine(f, hg.PREC_MIXED)
    assert e.check_mirror() == 0
    for _ in range(3):
        e.step(1)
        assert e.check_mirror() == 0
    e.autotune(steps=1)
    assert e.check_mirror() == 0
    e.fixup_bounds()
    assert e.check_mirror() == 0
    b = hg.Batch(0, 4)
    b.add(e)
    b.step()
    assert e.check_mirror() == 0
    b.remove(e)
    b.close()
    assert e.fail_counts().sum() > 0  # the stress state drives the fallback and fixup kernels
    e.close()


@pytest.mark.parametrize("kind,n", [("balsara", 1024), ("field_loop", 128)])
def test_mixed_keeps_transverse_components_zero(kind, n):
    """A shock tube along x1 and a field loop in the x1-x2 plane have U3 =
    B3 = 0 exactly in the FP64 form; every FP32 product that feeds them has
    an exact zero factor, so the mixed form must keep them exactly zero."""
    from coolharm3d_b200 import setups
    prob = setups.balsara1(n, precision=hg.PREC_MIXED) if kind == "balsara" else \
        setups.field_loop((n, n, 1), precision=hg.PREC_MIXED)
    e = hg.Engine(prob.desc)
    setups.start(e, prob)
    e.step(100)
    p = e.download()
    assert np.abs(p[..., 2:4]).max() > 0 or np.abs(p[..., 5:7]).max() > 0  # the flow evolved
    assert not p[..., 4].any() and not p[..., 7].any()
    assert e.check_mirror() == 0
    e.close()


@pytest.mark.parametrize("spacetime", [hg.DYN_MINK_SPHERICAL, hg.DYN_PN_BINARY])
def test_mixed_on_the_dynamic_metric_path(spacetime):
    """metric_dim 3: the FP32 fluxes read each time level's FP32 face
    geometry, written by the level kernel beside the FP64 one.  The binary
    disk (16x12x8) after 5 steps: relative L1 within 1e-5 of the FP64 run on
    every variable but the nearly-zero U1, U2 the flow only starts to
    develop (1e-3), finite, and not equal to it."""
    from coolharm3d_b200 import pnbbh
    n = (16, 12, 8)
    m = pnbbh.pnbbh_coords(spacetime=spacetime)
    out = {}
    p0 = None
    for prec in (hg.PREC_FP64, hg.PREC_MIXED):
        d = pnbbh.pnbbh_desc(n, precision=prec)
        t = pnbbh.pnbbh_tables(d)
        e = hg.Engine(d)
        e.set_dynamic_metric(m)
        e.set_cell_data(t["cell6"], t["rface"])
        e.set_cooling_tables(t["cool_omega"], t["cool_temp"])
        if p0 is None:
            p0, _ = pnbbh.set_disk(e, d, t, m)
        else:
            e.upload(p0)
        e.set_time(0.0, d.dx[0])
        e.step(5)
        out[prec] = e.download()
        e.close()
    p64, p32 = out[hg.PREC_FP64], out[hg.PREC_MIXED]
    assert np.isfinite(p32).all()
    err = l1_rel(p32, p64)
    print(spacetime, {k: "%.2e" % v for k, v in err.items()})
    assert max(v for k, v in err.items() if k not in ("U1", "U2")) < 1e-5, err
    assert max(err["U1"], err["U2"]) < 1e-3, err
    assert err != {k: 0.0 for k in NAMES}
