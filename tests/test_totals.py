"""dump_ener()'s integrals and the largest divb_calc() (hg_get_totals)
against the oracle's restatement of diag.c:503-612, 704-815 on the same
step."""
import numpy as np
import pytest

import coolharm3d_b200 as hg
import fixtures
import harmtest as ht
from test_gpu_parity import engine_for

CASES = ["linwave_noee_stress_10x8x6_s2", "linwave_12x10x8_s2", "balsara1_n128_s60", "torus_24x16x8_s3",
         "field_loop_24x24x1_s3"]


def oracle_after(f):
    o = ht.Oracle(f["n"], f["sw"], fixtures.geomd(f), lib=ht.CR_ORACLE)
    o.set_state(f["p0"], f["t0"], f["dt0"])
    o.step(f["steps"])
    return o


def test_oracle_mass_integral_is_m_tot():
    f = fixtures.load("linwave_12x10x8_s2")
    o = oracle_after(f)
    u, fl, dmax = o.totals()
    st = o.state()
    dV = f["dx"][1] * f["dx"][2] * f["dx"][3]
    assert u[0] == pytest.approx(st["m_tot"] * dV, rel=1e-13)
    assert dmax > 0  # the linear wave's analytic B is not corner-divergence-free; CT keeps what it has


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_totals_match_oracle(name):
    f = fixtures.load(name)
    e, _ = engine_for(f["n"], f["sw"], f, f["p0"], f["t0"], f["dt0"])
    e.step(f["steps"])
    u, fl, dmax = e.totals()
    uo, flo, dmo = oracle_after(f).totals()
    # sums of the same terms in another order: relative 1e-11, and for sums
    # that cancel to nearly nothing, 1e-14 of the largest integral
    np.testing.assert_allclose(u, uo, rtol=1e-11, atol=1e-14 * np.abs(uo).max())
    scale = np.abs(flo).max() + 1e-300
    assert np.abs(fl - flo).max() <= 1e-11 * scale, (fl, flo)
    assert dmax == pytest.approx(dmo, rel=1e-9, abs=1e-18)
    e.close()


@pytest.mark.gpu
def test_totals_survive_a_download_of_the_primitives():
    """The driver brings p back before diag() (and so dump_ener) runs: the
    boundary-flux integrals read after that download are the step's own."""
    f = fixtures.load("torus_24x16x8_s3")
    e, _ = engine_for(f["n"], f["sw"], f, f["p0"], f["t0"], f["dt0"])
    e.step(f["steps"])
    before = e.totals()
    e.download()
    e.pflag()
    e.gamma()
    after = e.totals()
    for a, b in zip(before, after):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    e.close()
