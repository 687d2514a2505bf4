"""Slab decomposition along z (mhy_b200/slabs.py) on the CPU with the oracle.

Each rank advances the oracle on its slab plus ghost layers; after every
cycle the dt minimum is combined over ranks and the ghost layers are
refreshed from the neighbours.  The owned layers of every rank must equal the
unsplit run bit for bit, over enough cycles to rotate the sweep order twice.
One test runs two ranks as processes over torch.distributed with gloo (the
code path bench.py uses with NCCL on GPUs); the others emulate the ranks in
one process.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import mhy_oracle
import slab_oracle
from mhy_b200 import gen, slabs

FIELDS = ("density", "internal_energy", "pressure", "sound_speed", "pseudo_viscosity", "cell_mass", "velocity",
          "node_mass")


def _reference(case, cycles):
    o = mhy_oracle.Oracle(case, threads=2)
    o.step(cycles)
    return o


def _check(case, ranks, ref):
    cl, nl = case.nx * case.ny, (case.nx + 1) * (case.ny + 1)
    for f in FIELDS:
        node = f in ("velocity", "node_mass")
        full = ref.field(f)
        for rk in ranks:
            s = rk.s
            lo = s.k0 * (nl if node else cl)
            hi = (s.k1 + (1 if node and s.rank == s.world - 1 else 0)) * (nl if node else cl)
            assert np.array_equal(rk.owned_field(f), full[lo:hi]), (f, s.rank)


def _split(case, world, ghost=slabs.GHOST):
    lay = slabs.layout(case.nz, world, ghost)
    return [slabs.SlabRank(case, lay, r, lambda c: slab_oracle.OracleEngine(c, mhy_oracle)) for r in range(world)]


@pytest.mark.parametrize("world", [2, 3])
def test_slabs_equal_the_unsplit_run(world):
    case = gen.sedov(n=20, jitter=0.01, seed=51, cycles=1) if world == 2 else \
        gen.sod(nx=6, ny=5, nz=30, lx=0.06, ly=0.05, lz=1.0, axis=2, jitter=0.01, seed=52, cycles=1)
    cycles = 9
    ranks = _split(case, world)
    slabs.run_local(ranks, cycles)
    _check(case, ranks, _reference(case, cycles))


@pytest.mark.parametrize("world,opts", [
    (2, {}),
    (3, {}),
    (2, dict(ordre_projection=3)),
    (2, dict(pente_borne=1, pente_borne_debar_fix=1)),
    (2, dict(conservation_energie_totale=1, projection_limiteur_id=5)),
], ids=["two", "three_ranks", "order3", "pente_borne", "cons_ec_g_limiter"])
def test_two_gas_slabs_equal_the_unsplit_run(world, opts):
    """Several environments: the ghost layers also carry the membership,
    every environment's values, the mixed/pure indicators and Phi."""
    case = gen.two_material(10, 6, 30 if world == 3 else 24, lx=0.5, ly=0.3, lz=1.2, seed=55, cycles=1,
                            options=gen.Options(**opts))
    cycles = 9
    ranks = _split(case, world)
    slabs.run_local(ranks, cycles)
    _check(case, ranks, _reference(case, cycles))


def test_ghost_depth_three_is_enough_and_two_is_not():
    """One cycle reaches at most 5 layers along z (the default depth); on this
    deck 3 ghost layers keep the split exact and 2 do not (the edge of the
    local mesh leaks into owned layers)."""
    case = gen.sedov(n=20, jitter=0.01, seed=53, cycles=1)
    ref = _reference(case, 6)
    ranks = _split(case, 2, ghost=3)
    slabs.run_local(ranks, 6)
    _check(case, ranks, ref)
    ranks = _split(case, 2, ghost=2)
    slabs.run_local(ranks, 6)
    with pytest.raises(AssertionError):
        _check(case, ranks, ref)


def test_layout_rules():
    lay = slabs.layout(40, 3)
    assert [(s.k0, s.k1, s.gb, s.gt) for s in lay] == [(0, 14, 0, 5), (14, 27, 5, 5), (27, 40, 5, 0)]
    with pytest.raises(ValueError):
        slabs.layout(10, 2)                  # 5 layers a slab: not more than the ghost depth


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    import pathlib
    root = pathlib.Path(__file__).resolve().parent.parent
    sys.path[:0] = [str(root / "arcane-benchs_b200"), str(root / "oracle"), str(root / "tests")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import mhy_oracle as orc
    import slab_oracle as so
    from mhy_b200 import gen as g, replicas, slabs as sl
    replicas.init("gloo", timeout_s=60)
    case = g.sedov(n=20, jitter=0.01, seed=54, cycles=1)
    lay = sl.layout(case.nz, world)
    rk = sl.SlabRank(case, lay, rank, lambda c: so.OracleEngine(c, orc))
    sl.run_distributed(rk, 7)
    q.put((rank, {f: rk.owned_field(f) for f in FIELDS}))
    dist.barrier()
    replicas.finish()


def test_two_rank_slabs_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    case = gen.sedov(n=20, jitter=0.01, seed=54, cycles=1)
    ref = _reference(case, 7)
    for f in FIELDS:
        got = np.concatenate([out[r][f] for r in range(2)])
        assert np.array_equal(got, ref.field(f)), f
