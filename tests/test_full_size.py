"""Parity at the benchmark's full size: the 192x192x128 magnetised torus
(Kerr-Schild a = 0.9, cooling, PPM_MC, HLLE, entropy fix, RESCALE_R), one
RK2 step of the engine against one step of the C oracle from the same
state (the build with the engine's correctly rounded pow(), see
tests/test_gpu_parity.py): bit-identical primitives, pflag, p_gamma and
counters in every zone, those repaired by the entropy fix included."""
import numpy as np
import pytest

import coolharm3d_b200 as hg
import harmtest as ht
from coolharm3d_b200 import torus
from test_gpu_parity import assert_same

pytestmark = pytest.mark.gpu

N = (192, 192, 128)
SW = dict(recon=hg.RECON_PPM_MC, flux=hg.FLUX_HLLE, ct_para=1, bc=hg.BC_SPHERICAL_OUTFLOW3, metric_dim=2, ee=1,
          cooling=1, rescale=1)


def test_full_size_torus_step_matches_oracle():
    d = torus.torus_desc(N)
    t = torus.torus_tables(d)
    e = hg.Engine(d)
    e.set_geometry(t["geom"], t["conn"])
    e.set_cell_data(t["cell6"], t["rface"])
    e.set_cooling_tables(t["cool_omega"], t["cool_temp"])
    p0 = torus.set_torus(e, d, t, seed=2024)
    o = ht.Oracle(N, SW, dict(gam=d.gam, cour=d.cour, grid_length=np.array(d.grid_length[:]),
                               startx=np.array(d.startx[:]), dx=np.array(d.dx[:]), geom=t["geom"], conn=t["conn"],
                               cell6=t["cell6"], rface=t["rface"], cool_omega=t["cool_omega"],
                               cool_temp=t["cool_temp"]), lib=ht.CR_ORACLE)
    o.set_state(p0, d.t, d.dx[0])
    e.set_time(d.t, d.dx[0])
    o.step(1)
    t1, dt1 = e.step(1)
    ref = o.state()
    ref["sw"] = SW
    assert (t1, dt1) == (ref["t"], ref["dt"])
    assert_same(e, ref, N)
    e.close()
