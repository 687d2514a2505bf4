"""GPU: the conservation-energie-totale remap option (RemapADI.axl:151,
RemapADIFinal.cc:751-773) in FP64, bit for bit against the oracle: Sod,
jittered Sedov, with schema-csts, order 3 and a stiffened gas; two and three
gases.

After the remap each cell's specific internal energy gains max(0, sum over its
8 nodes of 0.25 (U_dual[4] / U_dual[3] - 0.5 |v|^2)) times its mass fraction,
then p and c follow from the EOS.  The reference builds U_dual[4] as
0.5 m |v| (PrepareRemap.cc:421), not 0.5 m |v|^2, and that is kept, so the
option adds energy wherever |v| differs from |v|^2 (the oracle test
test_conservation_energie_totale_adds_energy states by how much).
"""
import numpy as np
import pytest

import mhy_oracle
from mhy_b200 import Batch, Context, MhyError, gen

pytestmark = pytest.mark.gpu

FIELDS = ("density", "internal_energy", "pressure", "sound_speed", "velocity", "node_mass", "cell_mass")


def _ec(case):
    case.options.conservation_energie_totale = 1
    return case


def _run(case, cycles):
    o = mhy_oracle.Oracle(case)
    g = Context(case)
    dto, dtg = [o.scalars()["dt"]], [g.dt()[0]]
    for _ in range(cycles):
        o.step(1)
        g.step(1)
        dto.append(o.scalars()["dt"])
        dtg.append(g.dt()[0])
    return o, g, dto, dtg


@pytest.mark.parametrize("make,cycles", [
    (lambda: gen.sod(cycles=120), 120),
    (lambda: gen.sedov(n=14, jitter=0.01, seed=31, cycles=60), 60),
    (lambda: gen.sod(nx=40, ny=6, nz=5, axis=1, lx=0.2, ly=1.0, lz=0.1, jitter=0.01, seed=32, cycles=60), 60),
])
def test_cons_ec_bitwise(make, cycles):
    case = _ec(make())
    o, g, dto, dtg = _run(case, cycles)
    assert dto == dtg
    for f in FIELDS:
        assert np.array_equal(o.field(f), g.field(f)), f
    assert g.kernels_per_cycle() == 11


@pytest.mark.parametrize("variant", ["csts", "order3", "stiffened", "newton", "entry_points"])
def test_cons_ec_with_other_options_bitwise(variant):
    case = _ec(gen.sedov(n=12, jitter=0.01, seed=33, cycles=40))
    if variant == "csts":
        case.options.schema_csts = 1
    elif variant == "order3":
        case.options.ordre_projection = 3
    elif variant == "stiffened":
        case.options.eos = (1,)
        case.options.limit_tension = (0.05,)
    elif variant == "newton":
        case.options.with_newton = 1
    o = mhy_oracle.Oracle(case)
    g = Context(case)
    o.step(40)
    if variant == "entry_points":
        for _ in range(40):
            g.cycle_by_entry_points()
    else:
        g.step(40)
    assert g.dt() == (o.scalars()["dt"], o.scalars()["old_dt"])
    for f in FIELDS:
        assert np.array_equal(o.field(f), g.field(f)), f


@pytest.mark.parametrize("make,cycles", [
    (lambda: gen.two_material(32, 16, 16, cycles=60, seed=9), 60),
    (lambda: gen.three_material(cycles=40), 40),
    (lambda: gen.two_material(24, 12, 12, cycles=40, seed=3, options=gen.Options(ordre_projection=3)), 40),
], ids=["two_gases", "three_gases", "two_gases_order3"])
def test_cons_ec_several_environments_bitwise(make, cycles):
    """Several environments: each environment's energy gains x_k delta, a
    mixed cell's mean gains delta, then every environment's EOS and the
    mixed-cell pressure and sound speed (RemapADIFinal.cc:751-773)."""
    case = _ec(make())
    o, g, dto, dtg = _run(case, cycles)
    assert dto == dtg
    for f in FIELDS:
        assert np.array_equal(o.field(f), g.field(f)), f
    for k in range(case.nenv):
        for w in ("fracvol", "density", "internal_energy"):
            assert np.array_equal(o.env_field(w, k), g.env_field(w, k)), (w, k)
    assert g.kernels_per_cycle() == (15 if case.options.ordre_projection == 3 else 12)


def test_cons_ec_refused_where_not_built():
    mixed = _ec(gen.sod(cycles=2))
    mixed.options.precision = 1
    with pytest.raises(MhyError):
        Context(mixed)
