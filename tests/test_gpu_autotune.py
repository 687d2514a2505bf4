"""GPU: the batch autotuner (mhy_batch_autotune) and explicit tunings.  Any
work order and persistent grid gives the same bits; autotuning restores the
batch state it trials on; a second batch with the same mesh sizes takes the
cached choice."""
import numpy as np
import pytest

from mhy_b200 import Batch, CTuning, MhyError, gen

pytestmark = pytest.mark.gpu

FIELDS = ("density", "internal_energy", "pressure", "velocity", "node_mass")


def cases():
    return gen.batched(count=6, seed=23, side_lo=8, side_hi=24, cycles=30)


def run(b, n):
    b.step(n)
    b.synchronize()
    return [{f: b.field(i, f) for f in FIELDS} | {"dt": b.dt(i)} for i in range(b.size())]


def assert_same(a, b):
    for i, (x, y) in enumerate(zip(a, b)):
        for f in FIELDS:
            assert np.array_equal(x[f], y[f]), (i, f)
        assert x["dt"] == y["dt"], i


def test_autotune_keeps_results_and_caches():
    ref = run(Batch(cases()), 30)
    b = Batch(cases())
    t = b.autotune(2)
    assert t.trials == 9 and not t.from_cache
    d = t.as_dict()["slots"]
    assert all(1 <= s["occupancy_pct"] <= 100 and s["ms_tuned"] > 0 for k, s in d.items() if k != "dt_finish")
    assert d["dt_min"]["order"] == d["lagrange_cells"]["order"]
    assert_same(ref, run(b, 30))
    t2 = Batch(cases()).autotune(2)
    assert t2.from_cache
    assert list(t2.order) == list(t.order) and list(t2.occupancy_pct) == list(t.occupancy_pct)


@pytest.mark.parametrize("order,pct", [(1, 100), (2, 50), (0, 25)])
def test_explicit_tunings_give_the_same_bits(order, pct):
    ref = run(Batch(cases()), 20)
    b = Batch(cases())
    t = CTuning()
    for k in range(10):
        t.order[k] = order
        t.occupancy_pct[k] = pct
    b.set_tuning(t)
    got = b.tuning()
    assert got.order[0] == order and got.occupancy_pct[3] == pct
    assert_same(ref, run(b, 20))


def test_bad_tuning_is_refused():
    b = Batch(cases())
    t = CTuning()
    for k in range(10):
        t.order[k] = 0
        t.occupancy_pct[k] = 100
    t.order[2] = 3
    with pytest.raises(MhyError):
        b.set_tuning(t)
    t.order[2] = 0
    t.occupancy_pct[5] = 0
    with pytest.raises(MhyError):
        b.set_tuning(t)
