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


def test_csr_structure_recovers_the_block_and_both_numberings():
    """mhy_csr_structure (host only) on a 7x5x4 block in a random cell and
    node numbering: the dimensions and the two maps come back exactly."""
    import numpy as np
    import pytest
    import csr_case
    from mhy_b200 import gen
    case = gen.sod(nx=7, ny=5, nz=4, cycles=1)
    s = csr_case.shuffled(case, seed=5)
    dims, ci, ni = mhy_b200.csr_structure(s["cell_nodes"], case.nnodes)
    assert dims == (7, 5, 4)
    assert np.array_equal(ci, s["cell_index"]) and np.array_equal(ni, s["node_index"])
    # the structured numbering itself maps to the identity
    dims, ci, ni = mhy_b200.csr_structure(csr_case.structured_cell_nodes(7, 5, 4), case.nnodes)
    assert dims == (7, 5, 4) and np.array_equal(ci, np.arange(case.ncells)) and np.array_equal(ni, np.arange(case.nnodes))
    # refused: a cell whose nodes are not in the SN_trigo order, a missing
    # cell, a node id out of range
    bad = s["cell_nodes"].copy()
    bad[3] = bad[3][[1, 2, 3, 0, 5, 6, 7, 4]]
    with pytest.raises(mhy_b200.MhyError) as e:
        mhy_b200.csr_structure(bad, case.nnodes)
    assert e.value.code == -4
    with pytest.raises(mhy_b200.MhyError) as e:
        mhy_b200.csr_structure(s["cell_nodes"][1:], case.nnodes)
    assert e.value.code == -4
    bad = s["cell_nodes"].copy()
    bad[0, 0] = case.nnodes
    with pytest.raises(mhy_b200.MhyError) as e:
        mhy_b200.csr_structure(bad, case.nnodes)
    assert e.value.code == -1


def test_options_default_matches_reference_defaults():
    mhy_b200.load()
    o = mhy_b200.COptions()
    mhy_b200.load().mhy_options_default(ctypes.byref(o))
    assert (o.cfl, o.threshold, o.deltat_init, o.deltat_min, o.deltat_max) == (0.3, 1e-10, 1e-5, 1e-8, 0.01)
    assert (o.ordre_projection, o.projection_limiteur_id, o.nb_bc) == (2, 0, 6)
