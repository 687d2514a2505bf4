"""GPU parity of the pente-borne remap (projection-pente-borne: Phi of
PrepareRemap.cc:201-212 and RemapADIService.cc:805-834, the general cell
gradient R:319-378, the fluxes of computeFluxPP / computeFluxPPPure
UtilesRemap.cc:406-823 with the reconstruction of :184-296 and INTY :83-93,
the debar fixes, face values R:574-578 and fluxes o*A*Phi_f R:770-774)
against the oracle, bit for bit; and the pure-neighbourhood limiter switch
of projection-pente-borne-mixte (R:369-375) on the default remap."""
import numpy as np
import pytest

import mhy_oracle
from mhy_b200 import Batch, Context, MhyError, gen

pytestmark = pytest.mark.gpu

FIELDS = ("density", "internal_energy", "velocity", "pressure", "pseudo_viscosity", "cell_mass", "node_mass",
          "sound_speed")
ERR_ARG, ERR_UNSUPPORTED = -1, -4


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


@pytest.mark.parametrize("debar", [0, 1, 2])
def test_pente_borne_sod_bitwise(debar):
    compare(gen.sod(cycles=150, options=gen.Options(pente_borne=1, pente_borne_debar_fix=debar)), 150, 30)


@pytest.mark.parametrize("limiter,debar", [(0, 1), (1, 2), (2, 1), (5, 2), (6, 1), (7, 0)])
def test_pente_borne_sedov_jittered_bitwise(limiter, debar):
    opts = gen.Options(pente_borne=1, pente_borne_debar_fix=debar, projection_limiteur_id=limiter)
    compare(gen.sedov(n=18, cycles=60, options=opts), 60, 20)


@pytest.mark.parametrize("pure_id,debar", [(1, 1), (2, 2), (4, 1), (0, 0)])
def test_pente_borne_mixte_pure_forms_bitwise(pure_id, debar):
    """One environment: every neighbourhood is pure, so the pure-cell fluxes
    (computeFluxPPPure) with projection-limiteur-pure-id apply, and the
    gradient takes that limiter when it is 1."""
    opts = gen.Options(pente_borne=1, pente_borne_mixte=1, limiteur_pure_id=pure_id, pente_borne_debar_fix=debar)
    compare(gen.sedov(n=16, cycles=50, options=opts), 50, 25)


def test_pente_borne_sod_along_z_with_newton_bitwise():
    case = gen.sod(nx=5, ny=5, nz=60, lx=0.05, ly=0.05, lz=1.0, axis=2, cycles=100,
                   options=gen.Options(pente_borne=1, pente_borne_debar_fix=1, with_newton=1))
    compare(case, 100, 25)


def test_pure_limiter_switch_without_pente_borne_bitwise():
    """projection-pente-borne-mixte alone: the default remap, with the cell
    gradients limited by superBee (limiteur-pure-id 1) while the dual ones
    keep projection-limiteur-id."""
    opts = gen.Options(pente_borne_mixte=1, limiteur_pure_id=1, projection_limiteur_id=2)
    compare(gen.sedov(n=18, cycles=60, options=opts), 60, 30)


def test_pente_borne_entry_points_match_graph():
    case = gen.sedov(n=14, cycles=30, options=gen.Options(pente_borne=1, pente_borne_debar_fix=1))
    a, b = Context(case), Context(case)
    for _ in range(30):
        a.cycle_by_entry_points()
    b.step(30)
    for f in ("density", "internal_energy", "velocity", "pseudo_viscosity"):
        assert np.array_equal(a.field(f), b.field(f)), f


def code_of(fn):
    with pytest.raises(MhyError) as ei:
        fn()
    return ei.value.code


@pytest.mark.parametrize("opts,code", [
    (dict(pente_borne=1, ordre_projection=1), ERR_UNSUPPORTED),
    (dict(pente_borne=1, ordre_projection=3), ERR_UNSUPPORTED),
    (dict(pente_borne=1, precision=1), ERR_UNSUPPORTED),
    (dict(pente_borne=1, pente_borne_debar_fix=3), ERR_ARG),
    (dict(pente_borne=2), ERR_ARG),
    (dict(pente_borne_mixte=1, limiteur_pure_id=8), ERR_ARG),
])
def test_unsupported_pente_borne_options_are_refused(opts, code):
    assert code_of(lambda: Context(gen.sod(cycles=1, options=gen.Options(**opts)))) == code


# Two gases (debar fix, projection-limiteur-id): the settings whose oracle run
# keeps a sane dt for 40 cycles.  With debar fix 0 an environment's mass flux
# lacks its volume fraction, and with pente-borne-mixte the pure cells keep
# that raw mass flux while an environment absent from a cell keeps the Phi of
# the previous remap (PrepareRemap.cc:201-212 sets only the cell's
# environments): there the oracle's dt collapses within a few cycles (to
# 1e-31 by cycle 2 for some settings), and the device follows it bit for bit.
SANE_FORMS = [(1, 0), (1, 1), (1, 5), (2, 2), (2, 6)]
# (debar fix, limiteur-pure-id, projection-limiteur-id) with pente-borne-mixte,
# run with deltat-min 0 for 10 cycles, during which the fields stay finite
MIXTE_FORMS = [(1, 1, 0), (1, 2, 5), (1, 4, 6), (2, 4, 2), (2, 1, 1), (0, 2, 1)]


@pytest.mark.parametrize("debar,limiter", SANE_FORMS)
def test_pente_borne_two_gases_bitwise(debar, limiter):
    """Several environments: Phi of PrepareRemap.cc:201-212 for the cell's
    environments (the others keep the last sweep's), every component's
    reconstruction and the debar fix over the environments."""
    opts = gen.Options(pente_borne=1, pente_borne_debar_fix=debar, projection_limiteur_id=limiter)
    compare(gen.two_material(32, 16, 16, cycles=40, seed=9, options=opts), 40, 10)


@pytest.mark.parametrize("debar,pure_id,limiter", MIXTE_FORMS)
def test_pente_borne_mixte_two_gases_bitwise(debar, pure_id, limiter):
    """pente-borne-mixte with two gases: the pure-neighbourhood choice cell
    by cell (limiters of the gradient and of the reconstruction, the mass
    flux left out of the debar fix), from the mixed/pure indicators of the
    previous remap on the first sweep and of the sweep's Phi afterwards."""
    opts = gen.Options(pente_borne=1, pente_borne_debar_fix=debar, pente_borne_mixte=1, limiteur_pure_id=pure_id,
                       projection_limiteur_id=limiter, deltat_min=0.0)
    compare(gen.two_material(32, 16, 16, cycles=10, seed=9, options=opts), 10, 2)


def test_pente_borne_debar0_two_gases_collapse_bitwise():
    """Debar fix 0 with two gases: the dt collapses (1e-17 at cycle 2) on both sides alike."""
    opts = gen.Options(pente_borne=1, pente_borne_debar_fix=0, deltat_min=0.0)
    compare(gen.two_material(32, 16, 16, cycles=4, seed=9, options=opts), 4, 2)


@pytest.mark.parametrize("debar", [1, 2])
def test_pente_borne_three_gases_bitwise(debar):
    compare(gen.three_material(cycles=30, options=gen.Options(pente_borne=1, pente_borne_debar_fix=debar)), 30, 10)


@pytest.mark.parametrize("limiter", [2, 5])
def test_pure_limiter_switch_two_gases_bitwise(limiter):
    """projection-pente-borne-mixte alone with two gases: superBee on the
    cells whose neighbourhood is pure, projection-limiteur-id elsewhere."""
    opts = gen.Options(pente_borne_mixte=1, limiteur_pure_id=1, projection_limiteur_id=limiter)
    compare(gen.two_material(32, 16, 16, cycles=40, seed=9, options=opts), 40, 20)


def test_pente_borne_two_gases_restart_dump():
    """The pente-borne Phi of absent environments and the mixed/pure
    indicators travel in the restart dump."""
    opts = gen.Options(pente_borne=1, pente_borne_debar_fix=1, pente_borne_mixte=1, limiteur_pure_id=2,
                       projection_limiteur_id=5, deltat_min=0.0)
    case = gen.two_material(32, 16, 16, cycles=10, seed=9, options=opts)
    a = Context(case)
    a.step(5)
    blob = a.save_checkpoint()
    b = Context.from_checkpoint(case, blob)
    a.step(5)
    b.step(5)
    for f in FIELDS:
        assert np.array_equal(a.field(f), b.field(f)), f


def test_pente_borne_in_some_batch_instances_is_refused():
    """A batch takes pente-borne in every instance or in none."""
    cases = gen.batched(count=2, seed=3, side_lo=8, side_hi=10, cycles=1)
    cases[1].options.pente_borne = 1
    assert code_of(lambda: Batch(cases)) == ERR_UNSUPPORTED


@pytest.mark.parametrize("opts", [
    dict(schema_csts=1),
    dict(eos=(1,), limit_tension=(0.5,)),
    dict(schema_csts=1, with_newton=0, projection_limiteur_id=1),
], ids=["csts", "stiffened", "csts_superbee"])
def test_pente_borne_with_other_options_bitwise(opts):
    """Pente-borne beside the schema-csts time scheme and the StiffenedGas EOS."""
    o = gen.Options(pente_borne=1, pente_borne_debar_fix=1, **opts)
    compare(gen.sod(cycles=120, options=o), 120, 30)
    compare(gen.sedov(n=14, cycles=40, options=gen.Options(pente_borne=1, pente_borne_debar_fix=2, **opts)), 40, 20)
