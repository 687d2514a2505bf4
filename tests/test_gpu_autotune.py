"""GPU: the autotuner (mhy_autotune, mhy_batch_autotune) and explicit
tunings.  Any lines per block of the y/z sweeps, work order and persistent
grid gives the same bits; autotuning restores the state it trials on; a
second context or batch with the same mesh sizes takes the cached choice."""
import numpy as np
import pytest

from mhy_b200 import Batch, Context, CTuning, MhyError, gen

pytestmark = pytest.mark.gpu

FIELDS = ("density", "internal_energy", "pressure", "velocity", "node_mass")


def cases():
    return gen.batched(count=6, seed=23, side_lo=8, side_hi=24, cycles=30)


def run(b, n):
    b.step(n)
    b.synchronize()
    return [{f: b.field(i, f) for f in FIELDS} | {"dt": b.dt(i)} for i in range(b.size())]


def run_ctx(g, n):
    g.step(n)
    g.synchronize()
    return [{f: g.field(f) for f in FIELDS} | {"dt": g.dt()}]


def assert_same(a, b):
    for i, (x, y) in enumerate(zip(a, b)):
        for f in FIELDS:
            assert np.array_equal(x[f], y[f]), (i, f)
        assert x["dt"] == y["dt"], i


def test_batch_autotune_keeps_results_and_caches():
    ref = run(Batch(cases()), 30)
    b = Batch(cases())
    t = b.autotune(2)
    assert t.trials == 27 and not t.from_cache
    d = t.as_dict()["slots"]
    assert all(1 <= s["occupancy_pct"] <= 100 and s["ms_tuned"] > 0 for k, s in d.items() if k != "dt_finish")
    assert d["dt_min"]["order"] == d["lagrange_cells"]["order"]
    assert all(d[k]["lines_per_block"] in (8, 16, 32) for k in ("cells_y", "cells_z", "nodes_y", "nodes_z"))
    assert_same(ref, run(b, 30))
    t2 = Batch(cases()).autotune(2)
    assert t2.from_cache
    assert list(t2.order) == list(t.order) and list(t2.lines_per_block) == list(t.lines_per_block)


@pytest.mark.parametrize("order,pct,lines", [(1, 100, 16), (2, 50, 32), (0, 25, 8)])
def test_batch_explicit_tunings_give_the_same_bits(order, pct, lines):
    ref = run(Batch(cases()), 20)
    b = Batch(cases())
    t = CTuning.default()
    for k in range(10):
        t.order[k] = order
        t.occupancy_pct[k] = pct
    for k in (3, 4, 6, 7):
        t.lines_per_block[k] = lines
    b.set_tuning(t)
    got = b.tuning()
    assert got.order[0] == order and got.occupancy_pct[3] == pct and got.lines_per_block[6] == lines
    assert_same(ref, run(b, 20))


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("lines", [16, 32])
def test_context_lines_per_block_give_the_same_bits(lines, precision):
    mk = lambda: gen.sedov(n=40, cycles=30, options=gen.Options(precision=precision))
    ref = run_ctx(Context(mk()), 30)
    g = Context(mk())
    t = CTuning.default()
    for k in (3, 4, 6, 7):
        t.lines_per_block[k] = lines
    g.set_tuning(t)
    assert_same(ref, run_ctx(g, 30))


def test_context_autotune_keeps_results_and_caches():
    mk = lambda: gen.sedov(n=36, cycles=30)
    ref = run_ctx(Context(mk()), 30)
    g = Context(mk())
    t = g.autotune(2)
    assert t.trials == 3 and not t.from_cache
    assert all(t.lines_per_block[k] in (8, 16, 32) for k in (3, 4, 6, 7))
    assert_same(ref, run_ctx(g, 30))
    assert Context(mk()).autotune(2).from_cache


def test_bad_tunings_are_refused():
    b = Batch(cases())
    t = CTuning.default()
    t.order[2] = 3
    with pytest.raises(MhyError):
        b.set_tuning(t)
    t = CTuning.default()
    t.occupancy_pct[5] = 0
    with pytest.raises(MhyError):
        b.set_tuning(t)
    t = CTuning.default()
    t.lines_per_block[2] = 16                     # the x sweeps keep 8 lines
    with pytest.raises(MhyError):
        b.set_tuning(t)
    g = Context(gen.two_material(16, 8, 8, cycles=5))
    t = CTuning.default()
    t.lines_per_block[3] = 16                     # K > 1 meshes keep 8 lines
    with pytest.raises(MhyError):
        g.set_tuning(t)
