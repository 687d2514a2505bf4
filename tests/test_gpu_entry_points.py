"""GPU: the per-entry-point C ABI records its work and launches it late (a
whole recorded cycle as one launch of the cycle graph; any call that reads
or waits on the device first launches what is pending).  Whatever the
interleaving of entry points and getters, the results are the bits of
mhy_step."""
import ctypes

import numpy as np
import pytest

import mhy_b200
from mhy_b200 import Context, gen

pytestmark = pytest.mark.gpu

ENTRY = ["mhy_save_values_at_n", "mhy_update_velocity", "mhy_apply_boundary_condition", "mhy_update_position",
         "mhy_compute_geometric_values", "mhy_update_density", "mhy_compute_artificial_viscosity",
         "mhy_update_energy_and_pressure", "mhy_remap", "mhy_compute_delta_t"]


def run_entries(g, cycles, probe_after=None):
    L = mhy_b200.load()
    for _ in range(cycles):
        for name in ENTRY:
            mhy_b200._check(getattr(L, name)(g.h))
            if probe_after == name:
                g.field("density")                   # reads the device mid-cycle: pending work launches first
                g.stream()


@pytest.mark.parametrize("probe", [None, "mhy_update_velocity", "mhy_compute_geometric_values", "mhy_remap"])
def test_entry_points_with_getters_match_step(probe):
    case = gen.sedov(n=16, cycles=20)
    ref = Context(case)
    ref.step(20)
    g = Context(case)
    run_entries(g, 20, probe)
    for f in ("density", "internal_energy", "velocity", "pressure", "node_mass"):
        assert np.array_equal(ref.field(f), g.field(f)), (probe, f)
    assert ref.dt() == g.dt() and ref.time() == g.time()


def test_entry_points_interleave_with_step():
    case = gen.two_material(16, 8, 8, cycles=12)
    ref = Context(case)
    ref.step(12)
    g = Context(case)
    run_entries(g, 4)
    g.step(4)
    run_entries(g, 4, "mhy_remap")
    for f in ("density", "internal_energy", "velocity"):
        assert np.array_equal(ref.field(f), g.field(f)), f
    assert np.array_equal(ref.env_mask(), g.env_mask())
