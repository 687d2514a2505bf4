"""GPU parity of the StiffenedGas equation of state
(eos/stiffenedgas/StiffenedGasEOSService.cc:10-44: e = (p + g pinf) /
((g-1) rho), p = (g-1) rho e - g pinf, c = sqrt(g/rho (p + pinf))) against
the oracle, bit for bit: one environment, two and three environments with
stiffened and perfect gases side by side, the batched form with a different
EOS per instance, the Newton energy update (with-newton), and the
mixed-precision form within its tolerance."""
import numpy as np
import pytest

import mhy_oracle
from mhy_b200 import Batch, Context, gen

pytestmark = pytest.mark.gpu

FIELDS = ("density", "internal_energy", "velocity", "pressure", "pseudo_viscosity", "cell_mass", "node_mass",
          "sound_speed")


def run_both(case, cycles, chunk):
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
    return o, g, np.array(dto), np.array(dtg)


def assert_bitwise(o, g, dto, dtg, K):
    assert np.array_equal(dto, dtg), f"dt sequences differ, first at {int(np.argmax(dto != dtg))}"
    for f in FIELDS:
        a, b = o.field(f), g.field(f)
        assert np.array_equal(a, b), f"{f}: {int((a != b).sum())} values differ"
    if K > 1:
        assert np.array_equal(o.env_mask(), g.env_mask())
        for k in range(K):
            for f in ("fracvol", "density", "internal_energy"):
                assert np.array_equal(o.env_field(f, k), g.env_field(f, k)), (k, f)
    assert g.status() == 0


def test_stiffened_sod_bitwise():
    case = gen.sod(cycles=200, options=gen.Options(eos=(1,), limit_tension=(0.5,)))
    o, g, dto, dtg = run_both(case, 200, chunk=25)
    assert_bitwise(o, g, dto, dtg, 1)
    # the stiffened branch ran: p + pinf = (g-1) rho e, not (g-1) rho e
    r, e, p = g.field("density"), g.field("internal_energy"), g.field("pressure")
    assert np.allclose(p, 0.4 * r * e - 1.4 * 0.5, rtol=0, atol=1e-12)


def test_stiffened_sedov_jittered_bitwise():
    case = gen.sedov(n=20, cycles=60, options=gen.Options(eos=(1,), limit_tension=(1.0e-3,)))
    o, g, dto, dtg = run_both(case, 60, chunk=20)
    assert_bitwise(o, g, dto, dtg, 1)


def test_two_material_one_stiffened_bitwise():
    opts = gen.Options(eos=(1, 0), limit_tension=(0.3, 0.0))
    case = gen.two_material(32, 16, 16, cycles=100, options=opts)
    o, g, dto, dtg = run_both(case, 100, chunk=10)
    assert_bitwise(o, g, dto, dtg, 2)


def test_three_material_mixed_eos_bitwise():
    opts = gen.Options(eos=(0, 1, 1), limit_tension=(0.0, 0.05, 0.2))
    case = gen.three_material(36, 12, 12, cycles=60, options=opts)
    o, g, dto, dtg = run_both(case, 60, chunk=15)
    assert_bitwise(o, g, dto, dtg, 3)


def test_batch_per_instance_eos_matches_single_contexts():
    cases = gen.batched(count=4, seed=41, side_lo=8, side_hi=16, cycles=30)
    cases[1].options.eos, cases[1].options.limit_tension = (1,), (0.2,)
    cases[2].options.eos, cases[2].options.limit_tension = (1,), (0.01,)
    b = Batch(cases)
    b.step(30)
    b.synchronize()
    for i, c in enumerate(cases):
        g = Context(c)
        g.step(30)
        for f in ("density", "internal_energy", "pressure", "velocity", "sound_speed"):
            assert np.array_equal(b.field(i, f), g.field(f)), (i, f)
        assert b.dt(i) == g.dt()


@pytest.mark.parametrize("deck", ["sod", "sod_stiffened", "sedov", "two_material"])
def test_newton_energy_update_bitwise(deck):
    """with-newton (MahycoModule.cc:1482-1535) on the device, bit for bit."""
    if deck == "sod":
        case = gen.sod(cycles=150, options=gen.Options(with_newton=1))
    elif deck == "sod_stiffened":
        case = gen.sod(cycles=150, options=gen.Options(with_newton=1, eos=(1,), limit_tension=(0.5,)))
    elif deck == "sedov":
        case = gen.sedov(n=20, cycles=60, options=gen.Options(with_newton=1))
    else:
        case = gen.two_material(32, 16, 16, cycles=80,
                                options=gen.Options(with_newton=1, eos=(1, 0), limit_tension=(0.3, 0.0)))
    o, g, dto, dtg = run_both(case, case.cycles, chunk=case.cycles // 4)
    assert_bitwise(o, g, dto, dtg, case.nenv)


@pytest.mark.parametrize("K", [1, 2])
def test_stiffened_mixed_precision_close_to_fp64(K):
    if K == 1:
        mk = lambda prec: gen.sod(cycles=200, options=gen.Options(eos=(1,), limit_tension=(0.5,), precision=prec))
    else:
        mk = lambda prec: gen.two_material(32, 16, 16, cycles=100,
                                           options=gen.Options(eos=(1, 0), limit_tension=(0.3, 0.0), precision=prec))
    a, b = Context(mk(0)), Context(mk(1))
    n = mk(0).cycles
    a.step(n)
    b.step(n)
    ra, rb = a.field("density"), b.field("density")
    l1 = float(np.abs(ra - rb).sum() / np.abs(ra).sum())
    assert l1 < 1.0e-5, l1
    ma, mb = a.field("cell_mass").sum(), b.field("cell_mass").sum()
    assert abs(ma - mb) <= 1e-11 * ma
