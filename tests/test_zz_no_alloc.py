"""The allocation-free time-step entry point, checked against the context's own dt.

mhy_compute_hydro_dt_noalloc is for callers that cannot call cudaMalloc: a
host framework that owns every device allocation (Arcane hands out its own
variables and memory pools), or code recording its work into a stream capture,
where allocation is not allowed.  Its scratch lives in a fixed __device__
array, so this test calls it through the C ABI on device buffers the test owns
and compares its dt, bit for bit like the other dt checks, with the dt that
mhy_compute_delta_t produced inside the context, on two consecutive cycles.

The file name makes pytest collect it last: a run that stops at the first
failure has executed every other test before this one.
"""
import numpy as np
import pytest

import mhy_b200
from mhy_b200 import Context, gen

pytestmark = pytest.mark.gpu


def _on_device(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to("cuda")


def test_noalloc_dt_equals_context_dt_on_two_calls():
    torch = pytest.importorskip("torch")
    case = gen.sedov(n=12, jitter=0.01, seed=21, cycles=2)
    ctx = Context(case, device=0)
    L = mhy_b200.load()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for call in range(2):
        ctx.step(1)
        ctx.synchronize()
        dt_new, dt_used = ctx.dt()
        lc = _on_device(torch, ctx.field("caracteristic_length"))
        cs = _on_device(torch, ctx.field("sound_speed"))
        v = _on_device(torch, ctx.field("velocity").T.copy())     # planes x[N], y[N], z[N]
        out.fill_(-1.0)
        torch.cuda.synchronize()
        rc = L.mhy_compute_hydro_dt_noalloc(case.nx, case.ny, case.nz, lc.data_ptr(), cs.data_ptr(), v.data_ptr(),
                                            case.options.cfl, dt_used, case.options.deltat_max, out.data_ptr(), None)
        assert rc == 0, f"call {call}: rc={rc}"
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[1] == dt_new, f"call {call}: no-alloc dt {got[1]!r} != context dt {dt_new!r}"
        assert got[0] > 0.0
    ctx.close()


def test_noalloc_rejects_meshes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    L = mhy_b200.load()
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    rc = L.mhy_compute_hydro_dt_noalloc(1024, 1024, 1024, p, p, p, 0.3, 1e-5, 0.01, p, None)
    assert rc == -1  # MHY_ERR_ARG: 2^30 cells exceed the 134217728-cell limit
