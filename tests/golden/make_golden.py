"""Golden fixtures of the oracle on small seeded cases.

The reference ships no golden data for this path, so these fixtures pin the
oracle (and, through the GPU tests, the device path) against regressions: the
final fields and the dt sequence of two small runs.  Regenerate with

    python tests/golden/make_golden.py

only when the oracle is deliberately changed, and commit the .npz files."""
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
for p in (ROOT / "arcane-benchs_b200", ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

import mhy_oracle  # noqa: E402
from mhy_b200 import gen  # noqa: E402

CASES = {
    "sod_small": lambda: gen.sod(nx=24, ny=4, nz=3, jitter=0.01, seed=4, cycles=40),
    "two_material_small": lambda: gen.two_material(16, 8, 8, cycles=30, seed=7),
    # option paths: pente-borne (debar fix 1, superBee); order 3 with a
    # generalised limiter, Newton energy update and a stiffened gas
    "sod_pente_borne_small": lambda: gen.sod(nx=24, ny=4, nz=3, jitter=0.01, seed=4, cycles=40, options=gen.Options(
        pente_borne=1, pente_borne_debar_fix=1, projection_limiteur_id=1)),
    "sedov_order3_options_small": lambda: gen.sedov(n=10, jitter=0.01, seed=9, cycles=25, options=gen.Options(
        ordre_projection=3, projection_limiteur_id=5, with_newton=1, eos=(1,), limit_tension=(1.0e-3,))),
}


def case(name):
    return CASES[name]()


def run(name):
    c = case(name)
    o = mhy_oracle.Oracle(c)
    dts = []
    for _ in range(c.cycles):
        dts.append(o.scalars()["dt"])
        o.step(1)
    dts.append(o.scalars()["dt"])
    out = {"dt": np.array(dts)}
    for f in ("density", "internal_energy", "pressure", "velocity", "node_mass"):
        out[f] = o.field(f)
    if c.nenv > 1:
        out["env_mask"] = o.env_mask()
        for k in range(c.nenv):
            out[f"fracvol_{k}"] = o.env_field("fracvol", k)
            out[f"density_{k}"] = o.env_field("density", k)
    return out


if __name__ == "__main__":
    # python tests/golden/make_golden.py [name ...]: all fixtures, or the named ones
    for name in (sys.argv[1:] or CASES):
        np.savez_compressed(HERE / f"{name}.npz", **run(name))
        print("wrote", HERE / f"{name}.npz")
