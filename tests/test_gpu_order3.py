"""GPU parity of the order-3 remap (ordre-projection 3: face values from
the six cells around each face, Remap-ordre-3.cc:7-131 with
RemapADIService.cc:583-641; cell widths RemapADIService.cc:225-258; the dual
remap's correction doubled by order2 = 2, DualPhaseRemap.cc:353) against the
oracle, bit for bit."""
import numpy as np
import pytest

import mhy_oracle
from mhy_b200 import Batch, Context, MhyError, gen

pytestmark = pytest.mark.gpu

FIELDS = ("density", "internal_energy", "velocity", "pressure", "pseudo_viscosity", "cell_mass", "node_mass",
          "sound_speed")


def compare(case, cycles, chunk):
    o, g = mhy_oracle.Oracle(case), Context(case)
    dto, dtg = [o.scalars()["dt"]], [g.dt()[0]]
    done = 0
    while done < cycles:
        n = min(chunk, cycles - done)
        o.step(n)
        g.step(n)
        done += n
        dto.append(o.scalars()["dt"])
        dtg.append(g.dt()[0])
    g.synchronize()
    assert np.array_equal(np.array(dto), np.array(dtg)), "dt sequences differ"
    for f in FIELDS:
        a, b = o.field(f), g.field(f)
        assert np.array_equal(a, b), f"{f}: {int((a != b).sum())} values differ"
    assert g.status() == 0


def test_order3_sod_bitwise():
    compare(gen.sod(cycles=150, options=gen.Options(ordre_projection=3)), 150, 30)


@pytest.mark.parametrize("limiter", [0, 2])
def test_order3_sedov_jittered_bitwise(limiter):
    opts = gen.Options(ordre_projection=3, projection_limiteur_id=limiter)
    compare(gen.sedov(n=20, cycles=80, options=opts), 80, 20)


def test_order3_sod_along_z_with_newton_bitwise():
    case = gen.sod(nx=5, ny=5, nz=60, lx=0.05, ly=0.05, lz=1.0, axis=2, cycles=100,
                   options=gen.Options(ordre_projection=3, with_newton=1))
    compare(case, 100, 25)


def test_order3_entry_points_match_graph():
    case = gen.sedov(n=14, cycles=30, options=gen.Options(ordre_projection=3))
    a, b = Context(case), Context(case)
    for _ in range(30):
        a.cycle_by_entry_points()
    b.step(30)
    for f in ("density", "internal_energy", "velocity"):
        assert np.array_equal(a.field(f), b.field(f)), f
    assert a.kernels_per_cycle() == 13


@pytest.mark.parametrize("limiter", [0, 2])
def test_order3_two_gases_bitwise(limiter):
    """Several environments: the face values of each component, then the
    density and energy rescaling on faces whose cells are not pure cells of
    one environment (R:623-641); the first sweep of the run sees every face
    as pure (the mixed/pure indicators start at zero)."""
    opts = gen.Options(ordre_projection=3, projection_limiteur_id=limiter)
    compare(gen.two_material(32, 16, 16, cycles=50, seed=9, options=opts), 50, 10)


def test_order3_three_gases_bitwise():
    compare(gen.three_material(cycles=40, options=gen.Options(ordre_projection=3)), 40, 10)


def test_order3_two_gases_entry_points_match_graph():
    case = gen.two_material(20, 10, 10, cycles=12, seed=4, options=gen.Options(ordre_projection=3))
    a, b = Context(case), Context(case)
    for _ in range(12):
        a.cycle_by_entry_points()
    b.step(12)
    for f in ("density", "internal_energy", "velocity"):
        assert np.array_equal(a.field(f), b.field(f)), f
    assert a.kernels_per_cycle() == 14


def test_order3_unsupported_forms_are_refused():
    with pytest.raises(MhyError):
        Context(gen.two_material(16, 8, 8, cycles=5, options=gen.Options(ordre_projection=3, precision=1)))
    with pytest.raises(MhyError):
        Context(gen.sod(cycles=5, options=gen.Options(ordre_projection=3, precision=1)))
    cases = gen.batched(count=2, seed=5, side_lo=8, side_hi=10, cycles=5)
    cases[0].options.ordre_projection = 3        # a batch takes order 3 in every instance or in none
    with pytest.raises(MhyError):
        Batch(cases)
