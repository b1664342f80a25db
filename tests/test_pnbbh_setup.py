"""Circumbinary-disk setup of the post-Newtonian binary runs
(coolharm3d_b200.pnbbh, restating init.nz_pn_bbh_disk.c) against the
reference's own initial state of that setup (reference configuration
pnbbh_dynmink: the dynamic-metric path with the Minkowski-spherical test
spacetime standing in for the PN metric, whose bodies the reference lacks).

The reference's perturbation comes from ranc() seeded with 1, so the whole
initial state -- disk, perturbed u, velocities through the grid metric,
normalised dipole loop, floors and boundaries -- is reproducible and is
compared bit for bit, as are the cooling tables its run uses.  On the CPU the
floors and boundaries come from the oracle (a metric_dim 2 target on one phi
slice of the axisymmetric stand-in metric); on the GPU from the engine, which
then steps the state and meets the reference's 3-step result."""
import numpy as np
import pytest

import coolharm3d_b200 as hg
import fixtures
import harmtest as ht
from coolharm3d_b200 import pnbbh

S1 = "pnbbh_dynmink_16x12x8_s1"
S3 = "pnbbh_dynmink_16x12x8_s3"


def grid(f):
    n = tuple(int(x) for x in f["n"])
    d = pnbbh.pnbbh_desc(n)
    return n, d, pnbbh.pnbbh_tables(d)


def oracle_target(f, n, t):
    T = [x + 2 * ht.NG for x in n]
    g3 = f["geom"].reshape(5, T[0], T[1], T[2], 42)
    geomd = dict(gam=f["gam"], cour=f["cour"], grid_length=f["grid_length"], startx=f["startx"], dx=f["dx"],
                 geom=np.ascontiguousarray(g3[:, :, :, 0].reshape(-1, 42)), conn=np.zeros((n[0] * n[1], 64)),
                 cell6=t["cell6"], rface=t["rface"], cool_omega=t["cool_omega"], cool_temp=t["cool_temp"])
    return ht.Oracle(n, dict(f["sw"], metric_dim=2), geomd)


def test_desc_matches_reference_grid():
    f = fixtures.load(S1)
    n, d, t = grid(f)
    np.testing.assert_array_equal(np.array(d.dx[:]), f["dx"])
    np.testing.assert_array_equal(np.array(d.startx[:]), f["startx"])
    np.testing.assert_array_equal(np.array(d.grid_length[:]), f["grid_length"])
    assert d.gam == f["gam"] and d.cour == f["cour"]
    sw = f["sw"]
    assert (d.recon_type, d.flux_type, d.use_flux_ct_para, d.bc_type, d.metric_dim, d.use_entropy_eq, d.cooling,
            d.rescale_r) == (sw["recon"], sw["flux"], sw["ct_para"], sw["bc"], sw["metric_dim"], sw["ee"],
                             sw["cooling"], sw["rescale"])
    np.testing.assert_array_equal(t["cell6"][..., :2], f["cell_floors"])
    np.testing.assert_array_equal(t["cell6"][:, ht.NG, ht.NG, 2], f["r_line"])
    np.testing.assert_array_equal(t["rface"], f["rface"])


def test_disk_matches_reference_initial_state_bit_for_bit():
    f = fixtures.load(S1)
    n, d, t = grid(f)
    p, h = pnbbh.set_disk(oracle_target(f, n, t), d, t, pnbbh.pnbbh_coords())
    assert h["inside"].any() and h["rho_max"] > 0
    for l in range(8):
        assert np.array_equal(p[..., l], f["p0"][..., l]), l


def test_cooling_tables_are_the_reference_runs():
    """The cooling tables and the RESCALE_R row the reference's run uses are
    the grid's own (the staged setup leaves the coordinates unshifted)."""
    f = fixtures.load(S1)
    n, d, t = grid(f)
    np.testing.assert_array_equal(t["cell6"][:, ht.NG, ht.NG, 3], f["x1_line"])
    np.testing.assert_array_equal(t["cool_omega"], f["cool_omega"])
    np.testing.assert_array_equal(t["cool_temp"], f["cool_temp"])


def test_ranc_is_reseeded():
    a, b, c = pnbbh.Ranc(1), pnbbh.Ranc(1), pnbbh.Ranc(2)
    xa = [a() for _ in range(100)]
    assert xa == [b() for _ in range(100)]
    assert xa != [c() for _ in range(100)]
    assert all(0.0 < x < 1.0 for x in xa)


@pytest.mark.gpu
def test_disk_on_engine_steps_like_the_reference():
    """The setup driven through the engine's floors and boundary kernels gives
    the reference's initial state bit for bit; three steps on the device's
    time-dependent metric path then meet the reference's 3-step state (the
    dynamic-metric bar: 1e-10 of each variable's largest magnitude, flags and
    counters exact)."""
    f3 = fixtures.load(S3)
    n, d, t = grid(f3)
    e = hg.Engine(d)
    m = pnbbh.pnbbh_coords()
    e.set_dynamic_metric(m)
    e.set_cell_data(t["cell6"], t["rface"])
    p0, h = pnbbh.set_disk(e, d, t, m)
    e.close()
    assert np.array_equal(p0, f3["p0"])
    # the reference's fixture run loads its initial state back (counters at
    # zero): so does a fresh engine here
    e = hg.Engine(d)
    e.set_dynamic_metric(m)
    e.set_cell_data(t["cell6"], t["rface"])
    e.set_cooling_tables(t["cool_omega"], t["cool_temp"])
    e.upload(p0)
    e.set_time(f3["t0"], f3["dt0"])
    e.step(f3["steps"])
    p = ht.interior(e.download(), n)
    r = ht.interior(f3["p"], n)
    scale = np.abs(r).reshape(-1, 8).max(0)
    d_rel = np.abs(p - r).reshape(-1, 8).max(0) / np.where(scale > 0, scale, 1.0)
    assert d_rel.max() <= 1e-10, d_rel
    assert np.array_equal(e.pflag(), f3["pflag"])
    assert e.fail_counts().tolist() == f3["nfailtot"].tolist()
    e.close()
