"""GPU: the autotuner (mhy_autotune, mhy_batch_autotune) and explicit
tunings.  Any lines per block of the y/z sweeps (one environment: 8, 16 or
32; the cell sweeps of several environments: 8 or 16), work order and
persistent grid gives the same bits; autotuning restores the state it trials on; a
second context or batch with the same mesh sizes takes the cached choice."""
import numpy as np
import pytest

from mhy_b200 import Batch, Context, CTuning, MhyError, gen

pytestmark = pytest.mark.gpu

FIELDS = ("density", "internal_energy", "pressure", "velocity", "node_mass")
ENV_FIELDS = ("fracvol", "density", "internal_energy")


def cases():
    return gen.batched(count=6, seed=23, side_lo=8, side_hi=24, cycles=30)


def run(b, n):
    b.step(n)
    b.synchronize()
    return [{f: b.field(i, f) for f in FIELDS} | {"dt": b.dt(i)} for i in range(b.size())]


def run_ctx(g, n, K=1):
    g.step(n)
    g.synchronize()
    env = {f"{f}{k}": g.env_field(f, k) for f in ENV_FIELDS for k in range(K)} if K > 1 else {}
    return [{f: g.field(f) for f in FIELDS} | env | {"dt": g.dt()}]


def assert_same(a, b):
    for i, (x, y) in enumerate(zip(a, b)):
        assert x.keys() == y.keys()
        for f in x:
            if f != "dt":
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


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("K", [2, 3])
def test_multi_environment_lines_per_block_give_the_same_bits(K, precision):
    """The cell y/z sweeps of several environments at 16 lines per block."""
    opts = gen.Options(precision=precision)
    mk = (lambda: gen.two_material(32, 20, 18, cycles=40, options=opts)) if K == 2 else \
         (lambda: gen.three_material(36, 17, 12, cycles=40, options=opts))
    ref = run_ctx(Context(mk()), 40, K)
    g = Context(mk())
    t = CTuning.default()
    t.lines_per_block[3] = t.lines_per_block[4] = 16
    g.set_tuning(t)
    assert list(g.tuning().lines_per_block)[3:5] == [16, 16]
    assert_same(ref, run_ctx(g, 40, K))


def test_multi_environment_autotune_keeps_results():
    mk = lambda: gen.two_material(40, 24, 24, cycles=30)
    ref = run_ctx(Context(mk()), 30, 2)
    g = Context(mk())
    t = g.autotune(2)
    assert t.trials == 2 and not t.from_cache
    assert all(t.lines_per_block[k] in (8, 16) for k in (3, 4))
    assert all(t.lines_per_block[k] == 8 for k in (0, 1, 2, 5, 6, 7))
    assert_same(ref, run_ctx(g, 30, 2))
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
    t.lines_per_block[3] = 32                     # several environments: cell y/z sweeps 8 or 16
    with pytest.raises(MhyError):
        g.set_tuning(t)
    t = CTuning.default()
    t.lines_per_block[6] = 16                     # and their node sweeps keep 8
    with pytest.raises(MhyError):
        g.set_tuning(t)
    g = Context(gen.sod(cycles=5, options=gen.Options(ordre_projection=3)))
    t = CTuning.default()
    t.lines_per_block[4] = 16                     # order 3 keeps 8 lines
    with pytest.raises(MhyError):
        g.set_tuning(t)
