"""The C-ABI library loads and exports every entry point declared in
include/harmgpu.h; host-side builders agree with the reference's tables.
No kernel runs here (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

import coolharm3d_b200 as hg
import fixtures
import harmtest as ht

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "harmgpu.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*\*?\s*(hg_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    lib = hg.load_library()
    names = declared()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(hg.EXPORTS) == names


def test_strerror_names_every_code():
    lib = hg.load_library()
    for code in range(0, -7, -1):
        assert lib.hg_strerror(code).decode() not in ("", "unknown error")
    assert lib.hg_strerror(-99).decode() == "unknown error"


def test_init_rejects_unsupported_switches():
    lib = hg.load_library()
    base = dict(n=(8, 8, 8), gam=4 / 3, cour=0.4, dx=[1e-5, .1, .1, .1], startx=[0, -.3, -.3, -.3],
                grid_length=[1, 1, 1, 1])
    bad = [dict(recon=7), dict(flux=3), dict(bc=5), dict(metric_dim=4), dict(metric_dim=3, n=(8, 8, 1)), dict(n=(0, 8, 8)),
           dict(metric_dim=2, n=(8, 1, 8)), dict(rescale_r=1, n=(1, 8, 8)), dict(gam=1.0),
           dict(n=(1290, 1290, 1290))]  # 2^31 entries per plane: past the kernels' 32-bit indexing
    for b in bad:
        kw = dict(base, **b)
        d = hg.make_desc(**kw)
        h = ctypes.c_void_p()
        assert lib.hg_init(ctypes.byref(d), ctypes.byref(h)) == -2, b
    assert lib.hg_init(None, ctypes.byref(ctypes.c_void_p())) == -2


@pytest.mark.parametrize("name", [n for n in fixtures.names() if "stress" not in n and not n.startswith("torus")])
def test_minkowski_builder_matches_reference_tables(name):
    f = fixtures.load(name)
    d = hg.make_desc(f["n"], f["gam"], f["cour"], f["dx"], f["startx"], f["grid_length"])
    geom, cell6 = hg.minkowski_tables(d)
    assert np.array_equal(geom, f["geom"][0])
    assert np.array_equal(np.signbit(geom), np.signbit(f["geom"][0]))
    assert np.array_equal(cell6[..., :2], f["cell_floors"])
