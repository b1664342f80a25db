"""restart_write()/restart_read() of the resident state (hg_write_rdump,
hg_read_rdump): the file is the reference's ASCII layout, field for field
what C's printf writes for the reference's formats (%28.18e, %14d), and a
state read back continues bit for bit."""
import numpy as np
import pytest

import coolharm3d_b200 as hg
import fixtures
from test_gpu_parity import engine_for

pytestmark = pytest.mark.gpu


def expected_text(p, n, t, gl0, nstep, gam, cour, n_out, rdump_cnt, dt):
    head = "%28.18e " % t + "".join("%14d " % x for x in n) + "%28.18e " % gl0 + "%14d " % nstep
    head += "%28.18e " % gam + "%28.18e " % cour + "".join("%14d " % x for x in n_out) + "%14d " % rdump_cnt
    head += "%28.18e " % dt + "\n"
    body = []
    for i in range(3, 3 + n[0]):
        for j in range(3, 3 + n[1]):
            for k in range(3, 3 + n[2]):
                body.append("".join("%28.18e " % v for v in p[i, j, k]) + "\n")
    return head + "".join(body)


@pytest.mark.parametrize("name", ["torus_24x16x8_s3", "balsara1_n128_s60"])
def test_rdump_layout_and_round_trip(name, tmp_path):
    f = fixtures.load(name)
    e, _ = engine_for(f["n"], f["sw"], f, f["p0"], f["t0"], f["dt0"])
    t, dt = e.step(2)
    p = e.download()
    n_out = np.arange(11, dtype=np.int32) * 3 + 1
    path = tmp_path / "rdump0.0000"
    e.write_rdump(path, nstep=2, n_out=n_out, rdump_cnt=5)
    text = path.read_text()
    want = expected_text(p, f["n"], t, f["grid_length"][0], 2, f["gam"], f["cour"], n_out, 5, dt)
    assert text == want
    # read back into a fresh grid: same state, same next steps
    e2, _ = engine_for(f["n"], f["sw"], f, f["p0"], f["t0"], f["dt0"])
    ns, no, rc = e2.read_rdump(path)
    assert (ns, rc) == (2, 5) and list(no) == list(n_out)
    np.testing.assert_array_equal(e2.download(), p)
    t1, dt1 = e.step(2)
    t2, dt2 = e2.step(2)
    assert (t1, dt1) == (t2, dt2)
    np.testing.assert_array_equal(e2.download(), e.download())
    e.close()
    e2.close()
