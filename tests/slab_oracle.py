"""The oracle as a slab engine (the shape of mhy_b200.slabs.GpuEngine), for
the CPU tests of the slab decomposition.  Test infrastructure only."""
import contextlib

class OracleEngine:
    """The CPU oracle on the local slab."""

    def __init__(self, case_local, oracle_module):
        self.o = oracle_module.Oracle(case_local)

    def on_stream(self):
        return contextlib.nullcontext()

    def set_dt_reduction(self, lo, hi):
        self.o.set_dt_reduction(lo, hi, True)

    def cycle(self):
        self.o.step(1)

    def local_min(self):
        import torch
        return torch.tensor([self.o.dt_local_min()], dtype=torch.float64)

    def finish(self, t):
        self.o.dt_finish(float(t[0]))

    def buffer(self, spec):
        import torch
        cl, ch, nl, nh = spec
        return torch.empty(self.o.halo_count(ch - cl, nh - nl), dtype=torch.float64)

    def pack(self, spec):
        import torch
        return torch.from_numpy(self.o.halo_pack(*spec))

    def unpack(self, spec, t):
        self.o.halo_unpack(*spec, t.numpy())

    def field(self, name):
        return self.o.field(name)

    def synchronize(self):
        pass

    def close(self):
        self.o.close()
