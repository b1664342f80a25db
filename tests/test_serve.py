"""Batches and the request server: a grid advanced inside a batch, among
other grids of other sizes and precisions, gives exactly the result it gets
alone (the same kernels run on it); the continuous-batching server returns,
for every request of a stream, the result the sequential server returns."""
import numpy as np
import pytest

import coolharm3d_b200 as hg
from coolharm3d_b200 import serve, setups

pytestmark = pytest.mark.gpu


def problems():
    return [setups.balsara1(128), setups.field_loop((32, 32, 1), precision=hg.PREC_MIXED),
            setups.linear_wave((16, 16, 16)), setups.balsara1(96, precision=hg.PREC_MIXED)]


def run_alone(prob, steps):
    e = hg.Engine(prob.desc)
    setups.start(e, prob)
    t, dt = e.step(steps)
    p = e.download()
    e.close()
    return p, t, dt


def test_batch_step_equals_alone():
    steps = 25
    probs = problems()
    engines = []
    b = hg.Batch(0, 8)
    for prob in probs:
        e = hg.Engine(prob.desc)
        setups.start(e, prob)
        b.add(e)
        engines.append(e)
    for s in range(steps):
        t, dt = b.step()
        if s == 10:  # member 1 leaves, takes one step alone, and joins again
            b.remove(engines[1])
            engines[1].step(1)
            b.add(engines[1])
    assert len(b) == 4
    for m, e in enumerate(engines):
        b.remove(e)
    b.close()
    for m, (e, prob) in enumerate(zip(engines, probs)):
        p, ta, dta = run_alone(prob, steps + (1 if m == 1 else 0))
        np.testing.assert_array_equal(e.download(), p)
        e.close()


def test_server_results_same_alone_and_in_mix():
    sizes = {"balsara1": (64, 128), "field_loop": (24, 32), "linear_wave": (12, 16)}
    stream = serve.make_stream(n=10, rate=1000.0, seed=7, time_scale=0.02, sizes=sizes)
    batched = serve.serve_batched(stream, max_slots=3, realtime=False, keep=True)
    seq = serve.serve_sequential(stream, realtime=False, keep=True)
    for a, s in zip(batched, seq):
        assert a.rid == s.rid and a.steps == s.steps and a.t == s.t, (a, s)
        np.testing.assert_array_equal(a.prims, s.prims)
        assert a.checksum == s.checksum
    summ = serve.summarize(batched)
    assert summ["requests"] == 10 and summ["p99_s"] >= summ["p50_s"] > 0


def _scaled_minkowski(geom, s):
    """Minkowski space in coordinates stretched by s: gcov = diag(-1, s^2, s^2, s^2)."""
    g = geom.copy()
    gcon, gcov = g[:16].reshape(4, 4), g[16:32].reshape(4, 4)
    for a in (1, 2, 3):
        gcov[a, a] = s * s
        gcon[a, a] = 1.0 / (s * s)
    g[32], g[33] = s ** 3, 1.0 / s ** 3
    return g


def test_member_changed_and_stepped_alone_is_recaptured_in_batch():
    """A member whose kernel arguments change (new geometry) and which then
    takes a step alone (recapturing its own step graph) must not be advanced
    by the batch's copy of its old graph: the batch rebuilds when a member's
    capture generation moved on."""
    prob = setups.linear_wave((12, 12, 12))
    geom0, _ = hg.minkowski_tables(prob.desc)
    geom1 = _scaled_minkowski(geom0, 1.1)
    a = hg.Engine(prob.desc)
    setups.start(a, prob)
    other = hg.Engine(setups.balsara1(64).desc)
    setups.start(other, setups.balsara1(64))
    b = hg.Batch(0, 4)
    b.add(a)
    b.add(other)
    for _ in range(3):
        b.step()
    a.set_geometry(geom1)
    a.step(1)          # recaptures a's own step graph with geom1
    for _ in range(2):
        b.step()       # must run a with geom1 too
    b.remove(a)
    b.remove(other)
    b.close()
    ref = hg.Engine(prob.desc)
    setups.start(ref, prob)
    ref.step(3)
    ref.set_geometry(geom1)
    ref.step(3)
    np.testing.assert_array_equal(a.download(), ref.download())
    for e in (a, other, ref):
        e.close()
