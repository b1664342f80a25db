"""The launch-configuration autotuner (hg_autotune): it leaves the resident
state as it found it, the configuration it picks is valid, and a step's
result does not depend on the launch configuration."""
import numpy as np
import pytest

import coolharm3d_b200 as hg
import fixtures
from test_gpu_parity import engine_for

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["torus_24x16x8_s3", "linwave_12x10x8_s2", "field_loop_24x24x1_s3"])
def test_autotune_keeps_state_and_results(name):
    f = fixtures.load(name)
    e, _ = engine_for(f["n"], f["sw"], f, f["p0"], f["t0"], f["dt0"])
    before = e.download()
    cfg, ms0, ms1 = e.autotune(steps=2)
    np.testing.assert_array_equal(e.download(), before)
    c = cfg.as_dict()
    assert 1 <= c["strip_faces"] <= 3 and c["strip_x1"] in (0, 1)
    assert all(c[k] >= 1 for k in ("grid_flux", "grid_flux32", "grid_emf", "grid_update", "grid_fixup", "grid_bounds"))
    assert ms1 <= ms0 * 1.0000001
    e.set_time(f["t0"], f["dt0"])
    t_tuned = e.step(f["steps"])
    p_tuned = e.download()
    ref, _ = engine_for(f["n"], f["sw"], f, f["p0"], f["t0"], f["dt0"])
    t_ref = ref.step(f["steps"])
    np.testing.assert_array_equal(p_tuned, ref.download())
    assert t_tuned == t_ref
    # every strip length gives the same step
    for nf, x1 in ((1, 1), (3, 0), (2, 1)):
        cfg2 = e.launch_config()
        cfg2.strip_faces = nf
        cfg2.strip_x1 = x1
        cfg2.grid_flux = 7
        e.set_launch_config(cfg2)
        e.upload(f["p0"])
        e.set_time(f["t0"], f["dt0"])
        e.step(f["steps"])
        np.testing.assert_array_equal(e.download(), p_tuned)
    e.close()
    ref.close()
