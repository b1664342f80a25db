"""The C oracle against golden fixtures made by the reference's own build.

Bit-identical primitives (every cell, ghosts included), pflag, p_gamma,
nfail, nfailtot, t, dx[0] and M_tot after the fixture's steps.
"""
import numpy as np
import pytest

import fixtures
import harmtest as ht


def oracle_for(f):
    return ht.Oracle(f["n"], f["sw"], fixtures.geomd(f))


@pytest.mark.parametrize("name", fixtures.names())
def test_oracle_matches_reference_fixture(name):
    f = fixtures.load(name)
    o = oracle_for(f)
    o.set_state(f["p0"], f["t0"], f["dt0"])
    o.step(f["steps"])
    s = o.state()
    n = f["n"]
    assert np.array_equal(s["p"], f["p"])
    assert np.array_equal(s["pflag"], f["pflag"])
    assert np.array_equal(ht.interior(s["gamma"], n), ht.interior(f["gamma"], n))
    assert np.array_equal(s["nfail"], f["nfail"])
    assert s["nfailtot"].tolist() == f["nfailtot"].tolist()
    assert s["t"] == f["t"] and s["dt"] == f["dt"]
    assert s["m_tot"] == f["m_tot"]


def test_stress_fixtures_exercise_every_fixup_branch():
    """The stress fixtures must drive the inversion fallbacks, the entropy fix,
    the gamma ceiling, floors and both interpolation fixups."""
    tot = np.zeros(ht.NFAIL, np.uint64)
    for name in fixtures.names():
        if "stress" in name:
            tot += fixtures.load(name)["nfailtot"]
    for slot in (0, 2, 4, 5, 6, 7, 8, 9):  # FLOOR GAMMA_MAX FULL_INV USE_EE UTOPRIM UTOPRIM_EE INTERP_PRIM INTERP_V
        assert tot[slot] > 0, slot
