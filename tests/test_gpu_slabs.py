"""GPU: the slab decomposition along z (mhy_b200/slabs.py) with device
contexts, its ranks emulated on one GPU in one process: each rank's context
runs its slab plus ghost layers, the host combines the dt minima and moves
the ghost layers between the contexts' device buffers (mhy_halo_pack /
mhy_halo_unpack).  The owned layers equal the unsplit context bit for bit in
FP64 and in the mixed form (whose corner vectors are FP32)."""
import numpy as np
import pytest

from mhy_b200 import Context, MhyError, gen, slabs

pytestmark = pytest.mark.gpu

FIELDS = ("density", "internal_energy", "pressure", "sound_speed", "pseudo_viscosity", "cell_mass", "velocity",
          "node_mass")


def _compare(case, world, cycles):
    lay = slabs.layout(case.nz, world)
    ranks = [slabs.SlabRank(case, lay, r, lambda c: slabs.GpuEngine(c, 0)) for r in range(world)]
    slabs.run_local(ranks, cycles)
    g = Context(case)
    g.step(cycles)
    cl, nl = case.nx * case.ny, (case.nx + 1) * (case.ny + 1)
    for f in FIELDS:
        node = f in ("velocity", "node_mass")
        full = g.field(f)
        got = np.concatenate([rk.owned_field(f) for rk in ranks])
        assert np.array_equal(got, full), f
    for rk in ranks:
        assert rk.eng.ctx.dt() == g.dt()
        rk.eng.close()


@pytest.mark.parametrize("world", [2, 3])
def test_gpu_slabs_equal_the_unsplit_context(world):
    case = gen.sedov(n=24, jitter=0.01, seed=61, cycles=1)
    _compare(case, world, 12)


def test_gpu_slabs_mixed_precision():
    case = gen.sod(nx=8, ny=6, nz=40, lx=0.08, ly=0.06, lz=1.0, axis=2, jitter=0.01, seed=62, cycles=1)
    case.options.precision = 1
    _compare(case, 2, 12)


@pytest.mark.parametrize("opts", [{}, dict(ordre_projection=3), dict(pente_borne=1, pente_borne_debar_fix=1)],
                         ids=["two_gases", "two_gases_order3", "two_gases_pente_borne"])
def test_gpu_slabs_two_gases(opts):
    """Several environments: the halo carries every environment plane of the
    restart state (membership, fractions, values, indicators, Phi)."""
    case = gen.two_material(10, 6, 24, lx=0.5, ly=0.3, lz=1.2, seed=55, cycles=1, options=gen.Options(**opts))
    lay = slabs.layout(case.nz, 2)
    ranks = [slabs.SlabRank(case, lay, r, lambda c: slabs.GpuEngine(c, 0)) for r in range(2)]
    slabs.run_local(ranks, 9)
    g = Context(case)
    g.step(9)
    for f in FIELDS:
        got = np.concatenate([rk.owned_field(f) for rk in ranks])
        assert np.array_equal(got, g.field(f)), f
    for k in range(case.nenv):
        for w in ("fracvol", "density", "internal_energy"):
            got = np.concatenate([slabs.owned(rk.s, rk.local, rk.eng.ctx.env_field(w, k), False) for rk in ranks])
            assert np.array_equal(got, g.env_field(w, k)), (w, k)
    for rk in ranks:
        rk.eng.close()


def test_halo_ranges_are_checked():
    g = Context(gen.sedov(n=8, cycles=1))
    with pytest.raises(MhyError):
        g.set_dt_reduction(3, 2)
    with pytest.raises(MhyError):
        g.halo_bytes(9, 0)
    assert g.halo_bytes(1, 1) == (6 + 24) * 8 * 64 + (3 + 1 + 3) * 8 * 81
