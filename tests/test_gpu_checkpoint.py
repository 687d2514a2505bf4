"""GPU: restart dumps (mhy_checkpoint_save / _load, the reference's
continue-init).  A run resumed from a dump taken between cycles continues
bit for bit like the uninterrupted run: one gas FP64, two gases, and the
mixed-precision form."""
import numpy as np
import pytest

from mhy_b200 import Context, MhyError, gen

pytestmark = pytest.mark.gpu

FIELDS = ("density", "internal_energy", "pressure", "velocity", "node_mass", "pseudo_viscosity")


def _mixed(c):
    c.options.precision = 1
    return c


@pytest.mark.parametrize("make", [
    lambda: gen.sedov(n=14, jitter=0.01, seed=2, cycles=60),
    lambda: gen.two_material(24, 12, 12, cycles=60, seed=9),
    lambda: gen.two_material(24, 12, 12, cycles=60, seed=9, options=gen.Options(ordre_projection=3)),
    lambda: _mixed(gen.sod(nx=40, ny=6, nz=5, jitter=0.01, seed=3, cycles=60)),
])
def test_resume_equals_uninterrupted_run(make):
    case = make()
    a = Context(case)
    a.step(25)                       # a dump between cycles, mid-way through a sens rotation
    a.cycle_by_entry_points()
    blob = a.save_checkpoint()
    a.step(20)
    b = Context.from_checkpoint(case, blob)
    assert b.dt() == pytest.approx(b.dt())
    b.step(20)
    assert a.dt() == b.dt() and a.time() == b.time()
    for f in FIELDS:
        assert np.array_equal(a.field(f), b.field(f)), f
    if case.nenv > 1:
        assert np.array_equal(a.env_mask(), b.env_mask())
        for k in range(case.nenv):
            assert np.array_equal(a.env_field("fracvol", k), b.env_field("fracvol", k))


def test_dump_of_another_mesh_is_rejected():
    a = Context(gen.sod(nx=20, ny=4, nz=4, cycles=5))
    a.step(2)
    blob = a.save_checkpoint()
    with pytest.raises(MhyError):
        Context.from_checkpoint(gen.sod(nx=22, ny=4, nz=4, cycles=5), blob)
    with pytest.raises(MhyError):
        Context.from_checkpoint(gen.sod(nx=20, ny=4, nz=4, cycles=5), b"garbage" * 10)


@pytest.mark.parametrize("change", ["limiter", "gamma", "newton", "eos", "cfl"])
def test_dump_with_other_physics_options_is_rejected(change):
    """The dump records a hash of the options that change the computed state;
    a context with the same mesh but other physics refuses it."""
    case = gen.sod(nx=20, ny=4, nz=4, cycles=5)
    a = Context(case)
    a.step(2)
    blob = a.save_checkpoint()
    other = gen.sod(nx=20, ny=4, nz=4, cycles=5)
    if change == "limiter":
        other.options.projection_limiteur_id = 1
    elif change == "gamma":
        other.gamma = np.array([1.5])
    elif change == "newton":
        other.options.with_newton = 1
    elif change == "eos":
        other.options.eos = (1,)
    else:
        other.options.cfl = 0.25
    with pytest.raises(MhyError):
        Context.from_checkpoint(other, blob)
    same = gen.sod(nx=20, ny=4, nz=4, cycles=5)
    same.options.deltat_init = 2e-5                     # replaced by the dump's dt: accepted
    b = Context.from_checkpoint(same, blob)
    assert b.dt() == a.dt()
