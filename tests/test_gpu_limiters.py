"""GPU parity of the generalised limiters for uneven cell widths
(projection-limiteur-id 3..7: minmodG, superBeeG, vanLeerG, arithmeticG,
ultrabeeG; fluxLimiterG, UtilesRemap.cc:127-175, on the cells through
RemapADIService.cc:319-437 and on the nodes through DualPhaseRemap.cc:48-64
and UtilesRemap.cc:15-80) against the oracle, bit for bit."""
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


@pytest.mark.parametrize("limiter", [3, 4, 5, 6, 7])
def test_g_limiter_sod_bitwise(limiter):
    compare(gen.sod(cycles=120, options=gen.Options(projection_limiteur_id=limiter)), 120, 40)


@pytest.mark.parametrize("limiter", [3, 5, 6])
def test_g_limiter_sedov_jittered_bitwise(limiter):
    compare(gen.sedov(n=18, cycles=60, options=gen.Options(projection_limiteur_id=limiter)), 60, 20)


def test_g_limiter_with_order3_and_csts_bitwise():
    compare(gen.sod(cycles=100, options=gen.Options(projection_limiteur_id=5, ordre_projection=3)), 100, 50)
    compare(gen.sedov(n=14, cycles=40, options=gen.Options(projection_limiteur_id=4, schema_csts=1)), 40, 20)


@pytest.mark.parametrize("limiter", [3, 4, 5, 6, 7])
def test_g_limiter_two_gases_bitwise(limiter):
    """Two ideal gases with a perturbed interface (mixed cells, membership
    changes): every remap component limited with the uneven-width limiter,
    the dual gradients with the dual widths."""
    compare(gen.two_material(32, 16, 16, cycles=50, seed=9, options=gen.Options(projection_limiteur_id=limiter)),
            50, 25)


def test_g_limiter_three_gases_bitwise():
    case = gen.three_material(cycles=40)
    case.options.projection_limiteur_id = 5
    compare(case, 40, 20)
    env_case = gen.two_material(24, 12, 12, cycles=30, seed=3, options=gen.Options(projection_limiteur_id=6))
    o, g = mhy_oracle.Oracle(env_case), Context(env_case)
    o.step(30)
    g.step(30)
    assert np.array_equal(o.env_mask(), g.env_mask())
    for k in range(2):
        assert np.array_equal(o.env_field("fracvol", k), g.env_field("fracvol", k))
        assert np.array_equal(o.env_field("density", k), g.env_field("density", k))


def test_g_limiter_unsupported_forms_are_refused():
    with pytest.raises(MhyError):
        Context(gen.sod(cycles=5, options=gen.Options(projection_limiteur_id=3, precision=1)))
    with pytest.raises(MhyError):
        Context(gen.sod(nx=20, ny=2, nz=2, cycles=5, options=gen.Options(projection_limiteur_id=3)))
    cases = gen.batched(count=2, seed=5, side_lo=8, side_hi=10, cycles=5)
    cases[1].options.projection_limiteur_id = 6
    with pytest.raises(MhyError):
        Batch(cases)
