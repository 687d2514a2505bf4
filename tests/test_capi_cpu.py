"""CPU-side checks of the C ABI library: it loads and exports every symbol include/mhy.h declares.

No compute call is made (there is no GPU on the build machine)."""
import ctypes
import pathlib
import re

import mhy_b200

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "mhy.h").read_text()
    return sorted(set(re.findall(r"\b(mhy_[a-z_0-9]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(mhy_b200.EXPORTED)


def test_library_exports_every_declared_symbol():
    import build  # arcane-benchs_b200/build.py
    build.build()
    lib = ctypes.CDLL(str(mhy_b200.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_options_default_matches_reference_defaults():
    mhy_b200.load()
    o = mhy_b200.COptions()
    mhy_b200.load().mhy_options_default(ctypes.byref(o))
    assert (o.cfl, o.threshold, o.deltat_init, o.deltat_min, o.deltat_max) == (0.3, 1e-10, 1e-5, 1e-8, 0.01)
    assert (o.ordre_projection, o.projection_limiteur_id, o.nb_bc) == (2, 0, 6)
