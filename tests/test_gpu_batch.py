"""GPU: the batched cycle (many uneven meshes in one set of persistent
launches, per-instance dt on the device; one, two or three gases) gives every
instance the bits of its own single-mesh run and of the oracle."""
import numpy as np
import pytest

import mhy_oracle
from mhy_b200 import Batch, Context, gen

pytestmark = pytest.mark.gpu

FIELDS = ("density", "internal_energy", "pressure", "velocity", "node_mass")


def small_batch():
    cases = gen.batched(count=6, seed=31, side_lo=8, side_hi=20, cycles=40)
    cases[1].options.projection_limiteur_id = 1                 # per-instance options
    cases[2].coords = gen.cartesian_nodes(cases[2].nx, cases[2].ny, cases[2].nz, 1.0, 1.0, 1.0, jitter=0.01, seed=5)
    for i, c in enumerate(cases):                              # per-instance dt from the first cycle on
        c.options.deltat_init = 1.0e-5 * (1 + i)
    cases[3].options.deltat_init = 5.0e-3                      # CFL-limited from the start
    return cases


def test_batch_matches_single_contexts_and_oracle():
    cases = small_batch()
    b = Batch(cases)
    dts_b = [[b.dt(i)[0]] for i in range(len(cases))]
    for _ in range(40):
        b.step(1)
        for i in range(len(cases)):
            dts_b[i].append(b.dt(i)[0])
    b.synchronize()
    assert b.kernels_per_cycle() == 10
    # every instance advances with its own dt
    assert len({d[-1] for d in dts_b}) == len(cases)
    for i, c in enumerate(cases):
        g = Context(c)
        o = mhy_oracle.Oracle(c)
        dts = [g.dt()[0]]
        for _ in range(40):
            g.step(1)
            o.step(1)
            dts.append(g.dt()[0])
        assert np.array_equal(np.array(dts), np.array(dts_b[i])), i
        for f in FIELDS:
            bf = b.field(i, f)
            assert np.array_equal(bf, g.field(f)), (i, f)
            assert np.array_equal(bf, o.field(f)), (i, f, "oracle")
        assert b.status(i) == 0


def test_batch_chunked_steps_equal_single_steps():
    cases = small_batch()
    a, b = Batch(cases), Batch(cases)
    for _ in range(10):
        a.step(3)
    b.step(30)
    for i in range(len(cases)):
        for f in FIELDS:
            assert np.array_equal(a.field(i, f), b.field(i, f)), (i, f)


def two_gas_batch(precision=0):
    cases = []
    for i, (nx, ny, nz) in enumerate([(16, 8, 8), (20, 10, 10), (12, 12, 6), (24, 8, 8)]):
        c = gen.two_material(nx, ny, nz, cycles=30, seed=40 + i)
        c.options.deltat_init = 1.0e-5 * (1 + i)
        c.options.precision = precision
        cases.append(c)
    cases[1].options.projection_limiteur_id = 1                 # per-instance options
    return cases


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_two_gases_matches_single_contexts(precision):
    """Instances with two environments each: the K-environment Lagrange
    kernel, cell sweeps, end-of-remap kernel and node sweeps over the batch's
    work tables give every instance the bits of its own context (and, in
    FP64, of the oracle)."""
    cases = two_gas_batch(precision)
    b = Batch(cases)
    b.step(30)
    b.synchronize()
    assert b.kernels_per_cycle() == 11
    for i, c in enumerate(cases):
        g = Context(c)
        g.step(30)
        assert b.dt(i) == g.dt(), i
        for f in FIELDS:
            assert np.array_equal(b.field(i, f), g.field(f)), (i, f)
        if precision == 0:
            o = mhy_oracle.Oracle(c)
            o.step(30)
            for f in FIELDS:
                assert np.array_equal(b.field(i, f), o.field(f)), (i, f, "oracle")
        assert b.status(i) == 0


def test_batch_three_gases_autotuned_matches_single_contexts():
    cases = [gen.three_material(nx=24, ny=8, nz=8, cycles=20), gen.three_material(nx=32, ny=12, nz=8, cycles=20)]
    b = Batch(cases)
    t = b.autotune(2)
    for k, w in enumerate(t.lines_per_block):
        assert w in ((8, 16) if k in (3, 4) else (8,)), (k, w)
    b.step(20)
    for i, c in enumerate(cases):
        g = Context(c)
        g.step(20)
        for f in FIELDS:
            assert np.array_equal(b.field(i, f), g.field(f)), (i, f)


def finite(b, i):
    return all(np.isfinite(b.field(i, f)).all() for f in FIELDS)


def _same_as_single_contexts(cases, cycles, oracle=True, sane=True):
    """Instance i of one batch equals a context of case i (dt, fields, status
    flags) and the oracle.  With sane=False an instance may raise a numeric
    status, provided its context raises the same one (NaN fields then compare
    equal where both sides hold NaN); the oracle, whose min/max treat NaN
    operands differently, checks only the instances that stayed finite."""
    b = Batch(cases)
    b.step(cycles)
    if sane:
        b.synchronize()
    for i, c in enumerate(cases):
        g = Context(c)
        g.step(cycles)
        assert b.status(i) == g.status(), i
        assert np.array_equal(b.dt(i), g.dt(), equal_nan=True), i
        for f in FIELDS:
            assert np.array_equal(b.field(i, f), g.field(f), equal_nan=True), (i, f)
        if oracle and (sane or finite(b, i)):
            o = mhy_oracle.Oracle(c)
            o.step(cycles)
            for f in FIELDS:
                assert np.array_equal(b.field(i, f), o.field(f), equal_nan=True), (i, f, "oracle")
        if sane:
            assert b.status(i) == 0
    return b


def test_batch_g_limiters_and_total_energy_match_single_contexts():
    """The G limiters in every instance (ids 3..7 per instance: the GL sweeps
    and the cell widths), conservation-energie-totale in some instances only
    (its kernel skips the others)."""
    cases = gen.batched(count=5, seed=33, side_lo=8, side_hi=16, cycles=25)
    for i, c in enumerate(cases):
        c.options.projection_limiteur_id = 3 + i % 5
        c.options.conservation_energie_totale = i % 2
    b = _same_as_single_contexts(cases, 25)
    assert b.kernels_per_cycle() == 11


def test_batch_two_gases_g_limiter_total_energy():
    cases = two_gas_batch()
    for i, c in enumerate(cases):
        c.options.projection_limiteur_id = 5 if i % 2 else 6
        c.options.conservation_energie_totale = 1 if i < 2 else 0
    b = _same_as_single_contexts(cases, 20)
    assert b.kernels_per_cycle() == 12


def test_batch_pente_borne_matches_single_contexts():
    """pente-borne in every instance (debar fix and limiters per instance;
    projection-pente-borne-mixte in some), one gas."""
    cases = gen.batched(count=5, seed=35, side_lo=8, side_hi=16, cycles=25)
    for i, c in enumerate(cases):
        c.options.pente_borne = 1
        c.options.pente_borne_debar_fix = 1 + i % 2
        c.options.projection_limiteur_id = (0, 1, 2, 1, 0)[i]
        c.options.pente_borne_mixte = i % 2
        c.options.limiteur_pure_id = 1
    b = _same_as_single_contexts(cases, 25)
    assert b.kernels_per_cycle() == 10


def test_batch_pente_borne_g_limiters_match_single_contexts():
    """pente-borne with a G limiter (ids 3..7) in every instance."""
    cases = gen.batched(count=5, seed=36, side_lo=8, side_hi=16, cycles=25)
    for i, c in enumerate(cases):
        c.options.pente_borne = 1
        c.options.pente_borne_debar_fix = 1 + i % 2
        c.options.projection_limiteur_id = 3 + i
        c.options.pente_borne_mixte = i % 2
        c.options.limiteur_pure_id = 4
    _same_as_single_contexts(cases, 25)


@pytest.mark.parametrize("mixte", [0, 1])
def test_batch_two_gases_pente_borne(mixte):
    cases = two_gas_batch()
    for i, c in enumerate(cases):
        c.options.pente_borne = 1
        c.options.pente_borne_debar_fix = 1 + i % 2
        c.options.pente_borne_mixte = mixte
        c.options.limiteur_pure_id = 2
        c.options.deltat_min = 0.0          # with -mixte two gases collapse (as in the oracle)
    b = _same_as_single_contexts(cases, 6 if mixte else 20, sane=not mixte)
    if mixte:   # the oracle keeps instances 0 and 2 finite over these cycles, 1 and 3 collapse
        assert [finite(b, i) for i in range(b.size())] == [True, False, True, False]


def test_batch_order3_matches_single_contexts():
    """Order 3 in every instance: the face kernel of each direction over the
    face work table, then the O3 cell sweeps (limiters and total energy per
    instance)."""
    cases = gen.batched(count=5, seed=37, side_lo=8, side_hi=16, cycles=25)
    for i, c in enumerate(cases):
        c.options.ordre_projection = 3
        c.options.projection_limiteur_id = (0, 1, 2, 1, 0)[i]
        c.options.conservation_energie_totale = i % 2
    b = _same_as_single_contexts(cases, 25)
    assert b.kernels_per_cycle() == 14


def test_batch_order3_g_limiters_match_single_contexts():
    cases = gen.batched(count=4, seed=38, side_lo=8, side_hi=14, cycles=20)
    for i, c in enumerate(cases):
        c.options.ordre_projection = 3
        c.options.projection_limiteur_id = 3 + i
    _same_as_single_contexts(cases, 20)


@pytest.mark.parametrize("limiter", [0, 5])
def test_batch_two_gases_order3(limiter):
    cases = two_gas_batch()
    for c in cases:
        c.options.ordre_projection = 3
        c.options.projection_limiteur_id = limiter
    b = _same_as_single_contexts(cases, 20)
    assert b.kernels_per_cycle() == 14


def test_batch_three_gases_order3():
    cases = [gen.three_material(cycles=15), gen.three_material(cycles=15)]
    cases[1].options.deltat_init = 2.0e-5
    for c in cases:
        c.options.ordre_projection = 3
    _same_as_single_contexts(cases, 15)


def test_batch_schema_csts_matches_single_contexts():
    """schema-csts in every instance: the CSTS cell kernel, the forward step
    over the node tiles and the face velocities over the face work table, the
    node sweeps on the Lagrangian coordinates (Newton and limiters per
    instance)."""
    cases = gen.batched(count=5, seed=39, side_lo=8, side_hi=16, cycles=25)
    for i, c in enumerate(cases):
        c.options.schema_csts = 1
        c.options.with_newton = i % 2
        c.options.projection_limiteur_id = (0, 1, 2, 1, 0)[i]
    b = _same_as_single_contexts(cases, 25)
    assert b.kernels_per_cycle() == 12


def test_batch_schema_csts_with_cell_widths():
    """schema-csts beside the G limiters, pente-borne and order 3 (the cell
    kernel's CSTS form with the cell widths)."""
    for extra in (dict(projection_limiteur_id=5), dict(pente_borne=1, pente_borne_debar_fix=1),
                  dict(ordre_projection=3)):
        cases = gen.batched(count=3, seed=40, side_lo=8, side_hi=12, cycles=15)
        for c in cases:
            c.options.schema_csts = 1
            for k, v in extra.items():
                setattr(c.options, k, v)
        _same_as_single_contexts(cases, 15)


def test_batch_two_gases_schema_csts():
    cases = two_gas_batch()
    for c in cases:
        c.options.schema_csts = 1
    b = _same_as_single_contexts(cases, 12)
    assert b.kernels_per_cycle() == 13


def test_batch_two_gases_pure_limiter_switch():
    cases = two_gas_batch()
    for c in cases:
        c.options.pente_borne_mixte = 1
        c.options.limiteur_pure_id = 1
        c.options.projection_limiteur_id = 2
    _same_as_single_contexts(cases, 20)
