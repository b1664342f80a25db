"""How much the reference's own step moves when pow() changes by one ulp.

pow() is correctly rounded neither in glibc nor in CUDA, and the entropy fix
(fixup.c:335-454, utoprim_1d_ee.c, utoprim_1d_ee2.c) feeds pow() results
into Newton solves.  This test rebuilds the C oracle with every pow() result
moved up by one ulp and measures the change after one step on the stress
fixtures: it is far above 1e-12.  This is why the engine does not use the
device's pow() there but hg_cr_pow, a correctly rounded pow() with the same
bits on host and device (tests/test_crpow.py): with it the engine matches the
reference bit for bit wherever glibc's pow() is correctly rounded, and pflag
and all failure counters must still agree exactly."""
import ctypes
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

import fixtures
import harmtest as ht

HOOK = "#include <math.h>\ndouble pow_ulp_up(double x, double y) { return nextafter(pow(x, y), INFINITY); }\n"


def _build_perturbed(td):
    hook = os.path.join(td, "hook.c")
    Path(hook).write_text(HOOK)
    so = os.path.join(td, "liboracle_powulp.so")
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-ffp-contract=off", "-shared", "-DOR_POW_HOOK=pow_ulp_up",
                           "-o", so, str(ht.REPO / "oracle" / "harm_oracle.c"), hook, "-lm"])
    return so


def _run(libpath, f):
    saved = (ht._olib, ht.ORACLE_SO)
    try:
        ht._olib, ht.ORACLE_SO = None, Path(libpath)
        shape = tuple(x + 6 for x in f["n"])
        cell6 = np.zeros(shape + (6,))
        cell6[..., :2] = f["cell_floors"]
        o = ht.Oracle(f["n"], f["sw"], fixtures.geomd(f, cell6))
        o.set_state(f["p0"], f["t0"], f["dt0"])
        o.step(1)
        return o.state()
    finally:
        ht._olib, ht.ORACLE_SO = saved


@pytest.mark.parametrize("name", ["balsara1_stress_n64_s1", "linwave_stress_10x8x6_s1"])
def test_one_ulp_of_pow_moves_entropy_fix_zones_beyond_1e12(name):
    f = fixtures.load(name)
    with tempfile.TemporaryDirectory() as td:
        a = _run(str(ht.ORACLE_SO), f)
        b = _run(_build_perturbed(td), f)
    d = np.abs(a["p"] - b["p"])
    sc = np.maximum(np.abs(a["p"]), np.abs(b["p"]))
    rd = np.where(d == 0, 0.0, d / np.where(sc > 0, sc, 1.0)).max()
    assert 1e-12 < rd < 1e-9
    assert np.array_equal(a["pflag"], b["pflag"])
    assert a["nfailtot"].tolist() == b["nfailtot"].tolist()
