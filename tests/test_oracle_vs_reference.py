"""The C oracle against a live run of the reference build (oracle/_ref).

Skipped where the reference build is absent (it is made by
oracle/build_ref.py from the reference sources)."""
import numpy as np
import pytest

import harmtest as ht

CASES = [("balsara1", (200, 1, 1), 40, None), ("balsara1_lf", (90, 1, 1), 25, None),
         ("linwave", (9, 7, 5), 3, 3), ("linwave_vl", (6, 6, 6), 2, 9), ("balsara1", (48, 1, 1), 3, 21),
         ("linwave", (1, 12, 10), 2, 4), ("linwave", (8, 1, 7), 2, 13), ("torus", (20, 12, 6), 4, "load"),
         ("torus", (12, 20, 4), 2, 31)]


def _sprinkle(p, seed):
    return _mg().sprinkle(p, seed)


def _mg():
    import importlib.util, os
    spec = importlib.util.spec_from_file_location(
        "mg", os.path.join(os.path.dirname(__file__), "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


def _stress(p, seed):
    import importlib.util, os
    spec = importlib.util.spec_from_file_location(
        "mg", os.path.join(os.path.dirname(__file__), "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.stress_state(p, seed)


@pytest.mark.parametrize("cfg,n,steps,seed", CASES)
def test_oracle_matches_live_reference(cfg, n, steps, seed):
    if not ht.ref_available(cfg):
        pytest.skip("reference build oracle/_ref/%s absent" % cfg)
    r0 = ht.run_ref(cfg, n, 1, dumps=[0], want_geom=True)
    s0 = r0["states"][0]
    if seed is None:
        load, p0, t0, dt0 = None, s0["p"], s0["t"], s0["dt"]
    elif seed == "load" or cfg == "torus":
        p0 = s0["p"] if seed == "load" else _sprinkle(s0["p"], seed)
        t0, dt0 = s0["t"], s0["dt"]
        load = dict(p=p0, t=t0, dt=dt0)
    else:
        p0, t0, dt0 = _stress(s0["p"], seed), s0["t"], 1e-4
        load = dict(p=p0, t=t0, dt=dt0)
    r = ht.run_ref(cfg, n, steps, load=load, dumps=range(1, steps + 1))
    o = ht.Oracle(n, ht.CONFIG_SWITCHES[cfg], r0["geom"])
    o.set_state(p0, t0, dt0)
    for s in range(1, steps + 1):
        o.step(1)
        a, b = o.state(), r["states"][s]
        assert np.array_equal(a["p"], b["p"]), s
        assert np.array_equal(a["pflag"], b["pflag"]), s
        assert np.array_equal(a["nfail"], b["nfail"]), s
        assert a["nfailtot"].tolist() == b["nfailtot"].tolist(), s
        assert a["dt"] == b["dt"] and a["t"] == b["t"], s
