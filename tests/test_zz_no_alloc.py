"""The allocation-free time-step entry point, checked against the context's own dt.

mhy_compute_hydro_dt_noalloc is for callers that cannot call cudaMalloc: a
host framework that owns every device allocation (Arcane hands out its own
variables and memory pools), or code recording its work into a stream capture,
where allocation is not allowed.  Its scratch lives in a fixed __device__
array, so this test calls it through the C ABI on device buffers the test owns
and compares its dt, bit for bit like the other dt checks, with the dt that
mhy_compute_delta_t produced inside the context, on two consecutive cycles;
once on a small mesh (one cell per thread) and once on a mesh above
8192 x 256 cells, where the first pass's grid is capped and each thread walks
several cells.  A field holding an invalid cell (negative length, NaN sound
speed) must not give a plausible dt: the call reports NaN and a zero dt.

The file name makes pytest collect it last: a run that stops at the first
failure has executed every other test before this one.
"""
import math

import numpy as np
import pytest

import mhy_b200
from mhy_b200 import Context, gen

pytestmark = pytest.mark.gpu


def _on_device(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to("cuda")


def _noalloc(L, case, lc, cs, v, dt_old, out):
    out.fill_(-1.0)
    import torch
    torch.cuda.synchronize()
    rc = L.mhy_compute_hydro_dt_noalloc(case.nx, case.ny, case.nz, lc.data_ptr(), cs.data_ptr(), v.data_ptr(),
                                        case.options.cfl, dt_old, case.options.deltat_max, out.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy().copy()


def _fields(torch, ctx):
    lc = _on_device(torch, ctx.field("caracteristic_length"))
    cs = _on_device(torch, ctx.field("sound_speed"))
    v = _on_device(torch, ctx.field("velocity").T.copy())     # planes x[N], y[N], z[N]
    return lc, cs, v


@pytest.mark.parametrize("n", [12, 130])
def test_noalloc_dt_equals_context_dt_on_two_calls(n):
    torch = pytest.importorskip("torch")
    case = gen.sedov(n=n, jitter=0.01, seed=21, cycles=2)
    ctx = Context(case, device=0)
    L = mhy_b200.load()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for call in range(2):
        ctx.step(1)
        ctx.synchronize()
        dt_new, dt_used = ctx.dt()
        lc, cs, v = _fields(torch, ctx)
        rc, got = _noalloc(L, case, lc, cs, v, dt_used, out)
        assert rc == 0, f"call {call}: rc={rc}"
        assert got[1] == dt_new, f"call {call}: no-alloc dt {got[1]!r} != context dt {dt_new!r}"
        assert got[0] > 0.0
    ctx.close()


def test_noalloc_reports_invalid_cells_then_recovers():
    torch = pytest.importorskip("torch")
    case = gen.sedov(n=12, jitter=0.01, seed=22, cycles=1)
    ctx = Context(case, device=0)
    L = mhy_b200.load()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    ctx.step(1)
    ctx.synchronize()
    dt_new, dt_used = ctx.dt()
    lc, cs, v = _fields(torch, ctx)
    bad_l = lc.clone()
    bad_l[777] = -abs(float(bad_l[777]))                        # an inverted cell
    rc, got = _noalloc(L, case, bad_l, cs, v, dt_used, out)
    assert rc == 0
    assert math.isnan(got[0]) and got[1] == 0.0, got
    bad_c = cs.clone()
    bad_c[5] = float("nan")                                      # a NaN field
    rc, got = _noalloc(L, case, lc, bad_c, v, dt_used, out)
    assert rc == 0
    assert math.isnan(got[0]) and got[1] == 0.0, got
    rc, got = _noalloc(L, case, lc, cs, v, dt_used, out)         # the shared scratch keeps no stale flag
    assert rc == 0 and got[1] == dt_new
    ctx.close()


def test_noalloc_rejects_meshes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    L = mhy_b200.load()
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    rc = L.mhy_compute_hydro_dt_noalloc(1024, 1024, 1024, p, p, p, 0.3, 1e-5, 0.01, p, None)
    assert rc == -1  # MHY_ERR_ARG: 2^30 cells exceed the 134217728-cell limit
