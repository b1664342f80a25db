"""The serving stream's batching bound (coolharm3d_b200.serve.stream_bound),
on made-up class rates: no GPU needed."""
import pytest

from coolharm3d_b200 import PREC_FP64, serve


def test_bound_is_the_ratio_of_alone_to_packed_time():
    st = [serve.Request(0, "balsara1", 512, PREC_FP64, 0.0), serve.Request(1, "field_loop", 512, PREC_FP64, 0.1)]
    cls = {("balsara1", 512, PREC_FP64): dict(dt=0.1, zones=512, t_final=1.0, alone=1e6, batched=1e8),
           ("field_loop", 512, PREC_FP64): dict(dt=0.5, zones=512 * 512, t_final=1.0, alone=5e8, batched=6e8)}
    b = serve.stream_bound(st, cls)
    w0, w1 = 512 * 10, 512 * 512 * 2
    assert b["max_speedup"] == pytest.approx((w0 / 1e6 + w1 / 5e8) / (w0 / 1e8 + w1 / 6e8))
    assert b["zone_update_share"]["field_loop"] == pytest.approx(w1 / (w0 + w1))
    assert sum(b["sequential_time_share"].values()) == pytest.approx(1.0)
