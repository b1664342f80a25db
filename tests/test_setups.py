"""Minkowski setups (coolharm3d_b200.setups) against the reference's own
initial states (init.balsara1.c, init.linearwave.c, init.field_loop.c run by
the reference build, tests/golden fixtures).  The setups' closing
fixup(p); bounds(p,0) comes from the oracle here; the GPU test drives the
engine."""
import numpy as np
import pytest

import coolharm3d_b200 as hg
import fixtures
import harmtest as ht
from coolharm3d_b200 import setups

# fixture, problem builder, tolerance (relative to each variable's scale)
CASES = [
    ("balsara1_n128_s1", lambda: setups.balsara1(128), 0.0),
    ("linwave_12x10x8_s2", lambda: setups.linear_wave((12, 10, 8)), 0.0),
    ("linwave_2d_16x16x1_s3", lambda: setups.linear_wave((16, 16, 1)), 0.0),
    ("field_loop_24x24x1_s3", lambda: setups.field_loop((24, 24, 1)), 0.0),
]


def oracle_for(prob, sw):
    d = prob.desc
    geomd = dict(gam=d.gam, cour=d.cour, grid_length=np.array(d.grid_length[:]), startx=np.array(d.startx[:]),
                 dx=np.array(d.dx[:]), geom=prob.geom, conn=np.zeros(1), cell6=prob.cell6, rface=None)
    return ht.Oracle(prob.n, sw, geomd)


@pytest.mark.parametrize("name,build,tol", CASES)
def test_setup_matches_reference_initial_state(name, build, tol):
    f = fixtures.load(name)
    prob = build()
    d = prob.desc
    np.testing.assert_array_equal(np.array(d.dx[:]), f["dx"])
    np.testing.assert_array_equal(np.array(d.startx[:]), f["startx"])
    np.testing.assert_allclose(np.array(d.grid_length[:]), f["grid_length"], rtol=1e-15)
    assert d.gam == f["gam"] and d.cour == f["cour"]
    sw = f["sw"]
    assert (d.recon_type, d.flux_type, d.use_flux_ct_para, d.bc_type) == (sw["recon"], sw["flux"], sw["ct_para"],
                                                                          sw["bc"])
    o = oracle_for(prob, sw)
    o.upload(prob.p_init)
    o.fixup_bounds()
    p = o.download()
    if tol == 0.0:
        bad = np.argwhere(p != f["p0"])
        assert bad.size == 0, (len(bad), bad[:4].tolist(), p[tuple(bad[0][:3])], f["p0"][tuple(bad[0][:3])])
    else:
        scale = np.abs(f["p0"]).max(axis=(0, 1, 2))
        assert (np.abs(p - f["p0"]).max(axis=(0, 1, 2)) <= tol * np.maximum(scale, 1e-300)).all()


@pytest.mark.gpu
@pytest.mark.parametrize("name,build,tol", CASES)
def test_setup_on_engine_matches_reference(name, build, tol):
    f = fixtures.load(name)
    prob = build()
    e = hg.Engine(prob.desc)
    setups.start(e, prob)
    p = e.download()
    np.testing.assert_array_equal(p, f["p0"])
    e.close()
