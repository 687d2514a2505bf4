"""GPU: contexts created from explicit connectivity (mhy_create_csr).

The same block in a random numbering of cells and nodes runs bit for bit like
the structured context, and every field comes back in the caller's numbering:
one gas (jittered Sedov) and two gases (per-environment fields and
membership).
"""
import numpy as np
import pytest

import csr_case
from mhy_b200 import Context, MhyError, gen

pytestmark = pytest.mark.gpu

CELL_FIELDS = ("density", "internal_energy", "pressure", "sound_speed", "pseudo_viscosity", "cell_mass",
               "cell_volume", "caracteristic_length")
NODE_FIELDS = ("velocity", "node_mass", "node_coord")


def _pair(case, seed):
    s = csr_case.shuffled(case, seed)
    g = Context(case)
    u = Context.from_csr(case, s["cell_nodes"], s["coords"], s["fracvol"], s["density"], s["pressure"],
                         s["velocity"])
    return s, g, u


@pytest.mark.parametrize("make,cycles", [
    (lambda: gen.sedov(n=12, jitter=0.01, seed=41, cycles=30), 30),
    (lambda: gen.two_material(24, 12, 12, cycles=30, seed=42), 30),
])
def test_csr_context_equals_structured_context(make, cycles):
    case = make()
    s, g, u = _pair(case, seed=7)
    ci, ni = s["cell_index"], s["node_index"]
    for f in NODE_FIELDS:                               # before any cycle: the caller's coordinates
        assert np.array_equal(u.field(f), g.field(f)[ni]), f
    g.step(cycles)
    u.step(cycles)
    assert u.dt() == g.dt()
    for f in CELL_FIELDS:
        assert np.array_equal(u.field(f), g.field(f)[ci]), f
    for f in NODE_FIELDS:
        assert np.array_equal(u.field(f), g.field(f)[ni]), f
    if case.nenv > 1:
        assert np.array_equal(u.env_mask(), g.env_mask()[ci])
        for k in range(case.nenv):
            for f in ("fracvol", "density", "internal_energy"):
                assert np.array_equal(u.env_field(f, k), g.env_field(f, k)[ci]), (f, k)


def test_csr_context_refuses_a_non_cartesian_block():
    case = gen.sedov(n=6, cycles=1)
    s = csr_case.shuffled(case, seed=3)
    cn = s["cell_nodes"].copy()
    cn[0] = cn[0][[4, 5, 6, 7, 0, 1, 2, 3]]             # one cell upside down
    with pytest.raises(MhyError) as e:
        Context.from_csr(case, cn, s["coords"], s["fracvol"], s["density"], s["pressure"], s["velocity"])
    assert e.value.code == -4
