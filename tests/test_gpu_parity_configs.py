"""GPU parity at the benchmark configurations' own sizes and cycle counts.

The other parity tests run small meshes; these run the stated workloads:

* Sedov 128^3 (1 % jitter, one ideal gas, FP64), 500 cycles, against the
  oracle evaluating V^(1/3.) with the C library's pow, as the reference does
  (MahycoModule.cc:1259, math::pow(V, 1./3.)).  Bar: density, specific
  internal energy and node velocity within 1e-10 relative L-infinity after
  the 500 cycles, and every dt of the sequence within 1e-12 relative.
* Two gases 256x128x128 (gamma 1.4 / 1.67, perturbed interface, mixed cells),
  60 cycles, bit for bit against the oracle with the project cube root on both
  sides: dt sequence, global fields, environment membership and the
  per-environment volume fractions and densities.

Each oracle run takes a few minutes on the host cores (the oracle is OpenMP).
"""
import numpy as np
import pytest

import mhy_oracle
from mhy_b200 import Context, gen

pytestmark = pytest.mark.gpu


def rel_linf(a, b):
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (scale if scale > 0 else 1.0))


def _run_recording_dt(case, cycles, pow_mode):
    o = mhy_oracle.Oracle(case, pow_mode=pow_mode)
    g = Context(case)
    dto, dtg = [o.scalars()["dt"]], [g.dt()[0]]
    for _ in range(cycles):
        g.step(1)
        dtg.append(g.dt()[0])                  # the dt the next cycle uses (device value, read each cycle)
    for _ in range(cycles):
        o.step(1)
        dto.append(o.scalars()["dt"])
    g.synchronize()
    return o, g, np.array(dto), np.array(dtg)


def test_sedov128_500_cycles_against_libm_oracle():
    case = gen.sedov(n=128)                    # the benchmark's mesh and state: 1 % jitter, seed 1
    o, g, dto, dtg = _run_recording_dt(case, 500, "libm")
    dt_err = float(np.max(np.abs(dtg - dto) / dto))
    errs = {f: rel_linf(g.field(f), o.field(f)) for f in ("density", "internal_energy", "velocity")}
    assert g.status() == 0
    assert dt_err <= 1e-12, f"dt sequence: max relative difference {dt_err:.3e}"
    for f, e in errs.items():
        assert e <= 1e-10, f"{f}: relative L-inf {e:.3e} after 500 cycles (all: {errs})"
    o.close()
    g.close()


def test_two_material_256x128x128_bitwise():
    cycles = 60
    case = gen.two_material(256, 128, 128, cycles=cycles)
    o, g, dto, dtg = _run_recording_dt(case, cycles, "project")
    assert np.array_equal(dto, dtg), f"dt sequences differ, first at {int(np.argmax(dto != dtg))}"
    for f in ("density", "internal_energy", "pressure", "velocity", "node_mass", "sound_speed"):
        a, b = o.field(f), g.field(f)
        assert np.array_equal(a, b), f"{f}: max rel diff {rel_linf(b, a):.3e}"
    assert np.array_equal(o.env_mask(), g.env_mask())
    for k in range(case.nenv):
        assert np.array_equal(o.env_field("fracvol", k), g.env_field("fracvol", k)), f"fracvol {k}"
        assert np.array_equal(o.env_field("density", k), g.env_field("density", k)), f"density {k}"
    o.close()
    g.close()
