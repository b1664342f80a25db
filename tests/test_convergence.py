"""The reference's linear slow-mode test (init.linearwave.c): after one wave
period the L1 error (final - initial state) falls with resolution.  The FP64
engine reproduces the reference's step bit for bit, so its order is the
reference's; the mixed-precision form must converge too, with errors within
a factor 2 of FP64's: its FP32 face fluxes round at 6e-8 of the background
state, which for this 1e-4 wave is not far below the truncation error, and
moves each error by up to 30% either way at these sizes."""
import pytest

import coolharm3d_b200 as hg
from coolharm3d_b200 import convergence

pytestmark = pytest.mark.gpu

SIZES = (16, 32, 64)


def test_linear_wave_converges_and_mixed_keeps_the_order():
    fp = convergence.study(sizes=SIZES, dims=2, precision=hg.PREC_FP64)
    mx = convergence.study(sizes=SIZES, dims=2, precision=hg.PREC_MIXED)
    print(fp["order"], mx["order"])
    for out in (fp, mx):
        errs = [e["rho"] for e in out["errors"]]
        assert errs[0] > errs[1] > errs[2] > 0
        for o in out["order"]:
            assert o["rho"] > 1.0 and o["B2"] > 1.0, o
    for a, b in zip(fp["errors"], mx["errors"]):
        for k in ("rho", "u", "U1", "U2", "B1", "B2"):
            assert 0.5 * a[k] <= b[k] <= 2.0 * a[k], (k, a[k], b[k])
