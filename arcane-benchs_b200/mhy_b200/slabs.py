"""One mesh split along z over several ranks: slabs with ghost layers.

The reference decomposes its mesh into MPI subdomains with ghost layers
(mahyco/src/MahycoModule.cc:62-75, 3 layers in mahyco/data/Data.512.arc) and
synchronises variables around its kernels; one cycle ends with a global
minimum for dt (ReducerMin, MahycoModule.cc:2067).  Here each rank holds an
ordinary context on its own z-slab plus `ghost` layers of each neighbour's
cells and nodes, deeper than one cycle's dependency reach along z, so one
exchange per cycle suffices and the owned layers of every rank come out of a
cycle exactly as in the unsplit run (the edge of the local mesh, with its
walls and boundary-plane rules, only corrupts ghost layers, which the next
exchange overwrites).  A cycle on rank r:

  1. the whole cycle on the local slab, the dt reduction restricted to the
     owned cell layers and stopped before the new dt;
  2. the minimum over ranks (all-reduce; the 64-bit pattern of a non-negative
     double orders like an integer, so the GPU reduces int64 bit patterns);
  3. the new dt from that minimum (identical on every rank);
  4. the ghost layers refreshed: the state every cycle starts from (the
     restart-dump fields) of the neighbours' owned boundary layers.

Engines: GpuEngine (a context on a GPU, buffers in device memory, collectives
over NCCL on the context's stream); the tests bring an engine of the same
shape around the CPU oracle for the world-size-2 gloo test.  run_distributed
drives one rank inside torch.distributed; run_local drives every rank of a
split in one process (bit-for-bit checks on one GPU).
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import gen

# Ghost layers per inner side: one cycle's dependency reach along z is at most
# 5 layers (Lagrange 1, cell sweep 2, node sweep with its mass fluxes 2); 3
# are enough on the test decks (2 are not), 5 are used.
GHOST = 5


@dataclasses.dataclass
class Slab:
    rank: int
    world: int
    k0: int      # owned global cell layers [k0, k1)
    k1: int
    gb: int      # ghost layers below (0 on the first rank)
    gt: int      # ghost layers above (0 on the last rank)

    @property
    def nz_local(self) -> int:
        return self.k1 - self.k0 + self.gb + self.gt

    @property
    def own(self) -> int:
        return self.k1 - self.k0

    # owned layers in local indices: cells [own_lo, own_hi); nodes the same,
    # plus the top node layer on the last rank
    @property
    def own_lo(self) -> int:
        return self.gb

    @property
    def own_hi(self) -> int:
        return self.gb + self.own

    @property
    def own_node_hi(self) -> int:
        return self.own_hi + (1 if self.rank == self.world - 1 else 0)


def layout(nz: int, world: int, ghost: int = GHOST) -> list[Slab]:
    """Owned cell layers as even as possible, lower ranks taking the extra
    layers; every slab must own more layers than a neighbour's ghost depth."""
    if world < 1:
        raise ValueError("world >= 1")
    base, extra = divmod(nz, world)
    out, k = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        if world > 1 and n < ghost + 1:
            raise ValueError(f"{nz} layers over {world} ranks: each slab needs at least {ghost + 1} layers")
        out.append(Slab(r, world, k, k + n, min(ghost, k), min(ghost, nz - (k + n))))
        k += n
    return out


def sub_case(case: gen.Case, s: Slab) -> gen.Case:
    """The rank's local mesh and initial state: cell layers [k0 - gb, k1 + gt)
    and node layers [k0 - gb, k1 + gt] of the global case."""
    cl, nl = case.nx * case.ny, (case.nx + 1) * (case.ny + 1)
    c0, c1 = (s.k0 - s.gb) * cl, (s.k1 + s.gt) * cl
    n0, n1 = (s.k0 - s.gb) * nl, (s.k1 + s.gt + 1) * nl
    return gen.Case(f"{case.name}-slab{s.rank}", case.nx, case.ny, s.nz_local, case.coords[n0:n1].copy(),
                    case.gamma, case.fracvol[:, c0:c1].copy(), case.density[:, c0:c1].copy(),
                    case.pressure[:, c0:c1].copy(), case.velocity[n0:n1].copy(), case.options, case.cycles)


def exchanges(slabs: list[Slab], r: int):
    """(sends, recvs) of rank r, each a list of (peer, (cell_lo, cell_hi,
    node_lo, node_hi)) in local layer indices, in a fixed order (down first)."""
    s = slabs[r]
    sends, recvs = [], []
    if r > 0:
        g = slabs[r - 1].gt                                 # the lower neighbour's upper ghost depth
        sends.append((r - 1, (s.own_lo, s.own_lo + g, s.own_lo, s.own_lo + g + 1)))
        recvs.append((r - 1, (0, s.gb, 0, s.gb)))
    if r < s.world - 1:
        g = slabs[r + 1].gb                                 # the upper neighbour's lower ghost depth
        sends.append((r + 1, (s.own_hi - g, s.own_hi, s.own_hi - g, s.own_hi)))
        recvs.append((r + 1, (s.own_hi, s.own_hi + s.gt, s.own_hi, s.own_hi + s.gt + 1)))
    return sends, recvs


def owned(s: Slab, case_local: gen.Case, values: np.ndarray, node: bool) -> np.ndarray:
    """The owned layers of a local cell (node) field, in global order."""
    if node:
        nl = (case_local.nx + 1) * (case_local.ny + 1)
        return values[s.own_lo * nl:s.own_node_hi * nl]
    cl = case_local.nx * case_local.ny
    return values[s.own_lo * cl:s.own_hi * cl]


class GpuEngine:
    """A context on one GPU; buffers are torch tensors in device memory,
    allocated and used on the context's own stream."""

    def __init__(self, case_local, device: int):
        import torch
        from . import Context
        self.torch = torch
        self.ctx = Context(case_local, device=device)
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.ExternalStream(self.ctx.stream(), device=self.dev)

    def on_stream(self):
        return self.torch.cuda.stream(self.stream)

    def set_dt_reduction(self, lo, hi):
        self.ctx.set_dt_reduction(lo, hi, True)

    def cycle(self):
        self.ctx.step(1)

    def local_min(self):
        with self.on_stream():
            t = self.torch.empty(1, dtype=self.torch.int64, device=self.dev)
            self.ctx.dt_local_min(t.data_ptr())
        return t

    def finish(self, t):
        with self.on_stream():
            self.ctx.dt_finish(t.data_ptr())

    def buffer(self, spec):
        cl, ch, nl, nh = spec
        with self.on_stream():
            return self.torch.empty(self.ctx.halo_bytes(ch - cl, nh - nl), dtype=self.torch.uint8, device=self.dev)

    def pack(self, spec):
        t = self.buffer(spec)
        with self.on_stream():
            self.ctx.halo_pack(*spec, t.data_ptr(), t.numel())
        return t

    def unpack(self, spec, t):
        with self.on_stream():
            self.ctx.halo_unpack(*spec, t.data_ptr(), t.numel())

    def field(self, name):
        return self.ctx.field(name)

    def synchronize(self):
        self.ctx.synchronize()

    def close(self):
        self.ctx.close()


class SlabRank:
    """Rank r of a split of `case`: its slab, local case and engine."""

    def __init__(self, case, slabs, r, make_engine):
        self.slabs, self.r, self.s = slabs, r, slabs[r]
        self.local = sub_case(case, self.s)
        self.eng = make_engine(self.local)
        self.eng.set_dt_reduction(self.s.own_lo, self.s.own_hi)
        self.sends, self.recvs = exchanges(slabs, r)

    def owned_field(self, name):
        node = name in ("velocity", "node_mass", "node_coord")
        return owned(self.s, self.local, self.eng.field(name), node)


def run_distributed(rank_obj: SlabRank, cycles: int):
    """cycles cycles of this rank inside torch.distributed (NCCL for GPU
    engines, gloo for the oracle); every rank calls it with the same count."""
    import torch.distributed as dist
    e = rank_obj.eng
    multi = dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1
    for _ in range(cycles):
        with e.on_stream():
            e.cycle()
            m = e.local_min()
            if multi:
                dist.all_reduce(m, op=dist.ReduceOp.MIN)
            e.finish(m)
            sent = [e.pack(spec) for _, spec in rank_obj.sends]
            got = [e.buffer(spec) for _, spec in rank_obj.recvs]
            reqs = [dist.isend(t, peer) for (peer, _), t in zip(rank_obj.sends, sent)]
            reqs += [dist.irecv(t, peer) for (peer, _), t in zip(rank_obj.recvs, got)]
            for q in reqs:
                q.wait()
            for (_, spec), t in zip(rank_obj.recvs, got):
                e.unpack(spec, t)
    e.synchronize()


def run_local(ranks: list[SlabRank], cycles: int):
    """Every rank of a split in one process, one after the other (the host
    orders all device work with explicit synchronisation; no rank waits on
    another inside a kernel)."""
    for _ in range(cycles):
        for rk in ranks:
            rk.eng.cycle()
        mins = [rk.eng.local_min() for rk in ranks]
        for rk in ranks:
            rk.eng.synchronize()
        m = mins[0].clone()
        for t in mins[1:]:
            m = m.minimum(t.to(m.device))
        if m.is_cuda:
            import torch
            torch.cuda.synchronize()                # m is read on the contexts' streams
        for rk in ranks:
            rk.eng.finish(m.to(mins[rk.r].device))
        packed = {}
        for rk in ranks:
            for peer, spec in rk.sends:
                packed[(rk.r, peer)] = rk.eng.pack(spec)
        for rk in ranks:
            rk.eng.synchronize()
        for rk in ranks:
            for peer, spec in rk.recvs:
                rk.eng.unpack(spec, packed[(peer, rk.r)])
        for rk in ranks:
            rk.eng.synchronize()
