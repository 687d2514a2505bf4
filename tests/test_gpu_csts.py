"""GPU parity of the schema-csts time scheme (Mahyco.axl:238; velocity taken
back to n-1/2 before the Lagrange step and forward to n+1 before the remap,
energy from the corner vectors of n and n+1: MahycoModule.cc:693-831,
1538-1613, 1776-1810, PrepareRemap.cc:69-79, 456) against the oracle, bit
for bit, with the closed-form and the Newton energy, through the cycle graph,
the entry points and a restart dump."""
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
    return g


@pytest.mark.parametrize("newton", [0, 1])
def test_csts_sod_bitwise(newton):
    compare(gen.sod(cycles=150, options=gen.Options(schema_csts=1, with_newton=newton)), 150, 30)


@pytest.mark.parametrize("newton", [0, 1])
def test_csts_sedov_jittered_bitwise(newton):
    compare(gen.sedov(n=20, cycles=80, options=gen.Options(schema_csts=1, with_newton=newton)), 80, 20)


def test_csts_stiffened_newton_bitwise():
    opts = gen.Options(schema_csts=1, with_newton=1, eos=(1,), limit_tension=(0.5,))
    compare(gen.sod(cycles=120, options=opts), 120, 40)


def test_csts_entry_points_and_restart_match_graph():
    case = gen.sedov(n=16, cycles=40, options=gen.Options(schema_csts=1))
    a, b = Context(case), Context(case)
    for _ in range(20):
        a.cycle_by_entry_points()
    b.step(20)
    blob = b.save_checkpoint()
    c = Context.from_checkpoint(case, blob)
    for _ in range(20):
        a.cycle_by_entry_points()
    b.step(20)
    c.step(20)
    for f in ("density", "internal_energy", "velocity", "pressure"):
        assert np.array_equal(a.field(f), b.field(f)), f
        assert np.array_equal(c.field(f), b.field(f)), f
    assert a.kernels_per_cycle() == 12


@pytest.mark.parametrize("newton", [0, 1])
def test_csts_two_gases_bitwise(newton):
    """Several environments: each environment's energy from the cell's
    corner-vector sums, and the forward step's p + q (a mixed cell's mean
    pressure of n plus sum_k f_k q_k)."""
    opts = gen.Options(schema_csts=1, with_newton=newton)
    compare(gen.two_material(32, 16, 16, cycles=50, seed=9, options=opts), 50, 10)


def test_csts_three_gases_bitwise():
    compare(gen.three_material(cycles=30, options=gen.Options(schema_csts=1, with_newton=1)), 30, 10)


def test_csts_two_gases_entry_points_and_restart_match_graph():
    case = gen.two_material(20, 10, 10, cycles=24, seed=4, options=gen.Options(schema_csts=1))
    a, b = Context(case), Context(case)
    for _ in range(12):
        a.cycle_by_entry_points()
    b.step(12)
    blob = b.save_checkpoint()
    c = Context.from_checkpoint(case, blob)
    for _ in range(12):
        a.cycle_by_entry_points()
    b.step(12)
    c.step(12)
    for f in ("density", "internal_energy", "velocity", "pressure"):
        assert np.array_equal(a.field(f), b.field(f)), f
        assert np.array_equal(c.field(f), b.field(f)), f
    assert a.kernels_per_cycle() == 13


def test_csts_unsupported_forms_are_refused():
    with pytest.raises(MhyError):
        Context(gen.two_material(16, 8, 8, cycles=5, options=gen.Options(schema_csts=1, precision=1)))
    with pytest.raises(MhyError):
        Context(gen.sod(cycles=5, options=gen.Options(schema_csts=1, precision=1)))
    cases = gen.batched(count=2, seed=5, side_lo=8, side_hi=10, cycles=5)
    cases[1].options.schema_csts = 1             # a batch takes schema-csts in every instance or in none
    with pytest.raises(MhyError):
        Batch(cases)
