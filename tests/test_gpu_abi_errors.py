"""GPU: the error behaviour of the C ABI (include/mhy.h): invalid options and
meshes are refused at mhy_create with MHY_ERR_ARG / MHY_ERR_UNSUPPORTED,
out-of-order entry points with MHY_ERR_ORDER (the time-loop order of
Mahyco.config:30-41), wrong buffer sizes with MHY_ERR_ARG, calls before
initialisation with MHY_ERR_STATE, and a dt below deltat-min with
MHY_ERR_DT_MIN and the status bit (the reference's exit(1),
MahycoModule.cc:2152-2159); the final time sets its status bit (the
reference's stopComputeLoop).  A refused call leaves a usable context."""
import ctypes

import numpy as np
import pytest

import mhy_b200
from mhy_b200 import Context, MhyError, gen

pytestmark = pytest.mark.gpu

ERR_ARG, ERR_UNSUPPORTED, ERR_ORDER, ERR_DT_MIN, ERR_STATE = -1, -4, -5, -6, -8


def code_of(fn):
    with pytest.raises(MhyError) as ei:
        fn()
    return ei.value.code


@pytest.mark.parametrize("field,value,code", [
    ("ordre_projection", 4, ERR_UNSUPPORTED),
    ("projection_limiteur_id", 9, ERR_UNSUPPORTED),
    ("precision", 2, ERR_ARG),
    ("with_newton", 3, ERR_ARG),
    ("schema_csts", 2, ERR_ARG),
    ("eos", (2,), ERR_ARG),
    ("cfl", -0.3, ERR_ARG),
])
def test_invalid_options_are_refused(field, value, code):
    opts = gen.Options(**{field: value})
    assert code_of(lambda: Context(gen.sod(cycles=1, options=opts))) == code


def test_invalid_mesh_and_gamma_are_refused():
    case = gen.sod(nx=1, ny=5, nz=5, lx=0.01, cycles=1)
    assert code_of(lambda: Context(case)) == ERR_ARG
    case = gen.sod(cycles=1, gamma=1.0)
    assert code_of(lambda: Context(case)) == ERR_ARG


def test_order_size_and_state_errors_leave_a_usable_context():
    case = gen.sedov(n=12, cycles=4)
    g = Context(case)
    L = mhy_b200.load()
    assert L.mhy_update_velocity(g.h) == ERR_ORDER                 # save_values_at_n must come first
    assert L.mhy_save_values_at_n(g.h) == 0
    assert L.mhy_remap(g.h) == ERR_ORDER
    assert L.mhy_step(g.h, 1) == ERR_ORDER                           # mid-cycle
    for name in ["mhy_update_velocity", "mhy_apply_boundary_condition", "mhy_update_position",
                 "mhy_compute_geometric_values", "mhy_update_density", "mhy_compute_artificial_viscosity",
                 "mhy_update_energy_and_pressure", "mhy_remap", "mhy_compute_delta_t"]:
        assert getattr(L, name)(g.h) == 0
    small = np.zeros(3)
    assert L.mhy_get_field(g.h, mhy_b200.FIELDS["density"], small.ctypes.data_as(ctypes.c_void_p), small.nbytes) == ERR_ARG
    assert L.mhy_step(g.h, -1) == ERR_ARG
    g.step(3)
    ref = Context(case)
    ref.step(4)
    assert np.array_equal(ref.field("density"), g.field("density"))
    h = Context(case, init=False)
    assert L.mhy_step(h.h, 1) == ERR_STATE
    out = (ctypes.c_double * 3)()
    assert L.mhy_get_totals(h.h, out) != 0


def test_dt_min_and_final_time():
    opts = gen.Options(deltat_min=1.0)                 # any CFL dt is below it
    g = Context(gen.sod(cycles=3, options=opts))
    g.step(2)
    assert code_of(g.synchronize) == ERR_DT_MIN
    assert g.status() & 0x1
    opts = gen.Options(final_time=1.0e-4)
    g = Context(gen.sod(cycles=30, options=opts))
    g.step(30)
    g.synchronize()
    assert g.status() & 0x2
