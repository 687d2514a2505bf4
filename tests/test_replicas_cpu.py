"""The multi-GPU host logic of bench.py (replicas, barrier, max over ranks)
with world size 2 on the gloo backend, each rank advancing its own oracle
mesh on the CPU in place of a GPU replica."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    import time
    import pathlib
    root = pathlib.Path(__file__).resolve().parent.parent
    sys.path[:0] = [str(root / "arcane-benchs_b200"), str(root / "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from mhy_b200 import gen, replicas
    import mhy_oracle
    replicas.init("gloo", timeout_s=60)
    w, r, _ = replicas.ranks()
    case = gen.sod(nx=20 + 10 * r, ny=4, nz=4, cycles=3)        # uneven replicas
    o = mhy_oracle.Oracle(case, threads=1)
    replicas.barrier()
    t0 = time.perf_counter()
    o.step(3)
    ms = (time.perf_counter() - t0) * 1e3
    replicas.barrier()
    ms_max, value = replicas.aggregate(case.ncells, 3, ms)
    q.put((r, w, ms, ms_max, value, case.ncells))
    replicas.finish()


def test_two_rank_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    ms = [o[2] for o in out]
    for r, w, _, ms_max, value, cells in out:
        assert w == 2
        assert ms_max == pytest.approx(max(ms))
        # whole-job figure: both ranks' units over the slowest time
        assert value == pytest.approx((out[0][5] + out[1][5]) * 3 / (ms_max / 1e3))


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_batched_instances_partition_by_cells(world):
    """The batched workload's split over ranks: every instance on exactly one
    rank, the same split whichever rank computes it, and the heaviest rank
    within 1 % of the mean load (round-robin: up to 1.39x at 8 ranks)."""
    from mhy_b200 import gen, replicas
    cells = [c.ncells for c in gen.batched()]
    parts = [replicas.partition(cells, world, r) for r in range(world)]
    assert sorted(i for p in parts for i in p) == list(range(len(cells)))
    assert all(p == sorted(p) for p in parts)
    assert parts == [replicas.partition(cells, world, r) for r in range(world)]
    loads = [sum(cells[i] for i in p) for p in parts]
    assert max(loads) <= 1.01 * sum(cells) / world
    with pytest.raises(ValueError):
        replicas.partition(cells, world, world)
