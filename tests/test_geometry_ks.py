"""Host builder of the Kerr-Schild / modified Kerr-Schild tables
(hg_build_geometry_ks_mks) against the tables the reference's own build
computed for the torus fixtures (calc_all_geom, metric.c:4111-4265, and the
H/R cooling tables of phys.c:805-905).  No GPU: the builder is host code."""
import numpy as np
import pytest

import coolharm3d_b200 as hg
import fixtures

TORUS = [n for n in fixtures.names() if n.startswith("torus")]


def rel(a, b):
    scale = np.maximum(np.abs(a), np.abs(b))
    return np.where(scale > 0, np.abs(a - b) / np.where(scale > 0, scale, 1.0), 0.0)


def tables_for(f):
    d = hg.make_desc(f["n"], f["gam"], f["cour"], f["dx"], f["startx"], f["grid_length"], metric_dim=2,
                     bc=hg.BC_SPHERICAL_OUTFLOW3, cooling=1,
                     rescale_r=1)
    return hg.ks_mks_tables(d, a=0.9, h_o_r=0.1)


@pytest.mark.parametrize("name", TORUS)
def test_ks_mks_builder_matches_reference_tables(name):
    f = fixtures.load(name)
    t = tables_for(f)
    # metric, inverse, determinant, lapse, shift, normal observer: to rounding
    assert t["geom"].shape == f["geom"].shape
    assert rel(t["geom"], f["geom"]).max() < 1e-11
    # connection: complex-step derivatives vs the reference's closed form
    scale = np.abs(f["conn"]).max()
    assert np.abs(t["conn"] - f["conn"]).max() < 1e-14 * scale
    # floors, radii and the cooling tables are formed the same way: exact
    np.testing.assert_array_equal(t["cell6"][..., :2], f["cell_floors"])
    np.testing.assert_array_equal(t["cell6"][:, 3, 3, 2], f["r_line"])
    np.testing.assert_array_equal(t["rface"], f["rface"])
    np.testing.assert_array_equal(t["cool_omega"], f["cool_omega"])
    np.testing.assert_array_equal(t["cool_temp"], f["cool_temp"])


def test_ks_mks_builder_rejects_bad_spin():
    f = fixtures.load(TORUS[0])
    d = hg.make_desc(f["n"], f["gam"], f["cour"], f["dx"], f["startx"], f["grid_length"], metric_dim=2)
    with pytest.raises(hg.HarmGPUError):
        hg.ks_mks_tables(d, a=1.0)
