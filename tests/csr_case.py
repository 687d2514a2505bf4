"""A generated case re-expressed as explicit connectivity in a random numbering.

Used by the explicit-connectivity tests: the structured block of a case gets a
random permutation of its cells and of its nodes, as a mesh file or another
framework's item numbering would present it.
"""
import numpy as np

# SN_trigo node offsets of a hexahedral cell (cartesian/CartConnectivityCellNode.h:83-94)
OFF = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])


def structured_cell_nodes(nx, ny, nz):
    """(C, 8) structured node ids of every structured cell."""
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    return np.stack([(i + o[0]) + (nx + 1) * ((j + o[1]) + (ny + 1) * (k + o[2])) for o in OFF], axis=1)


def shuffled(case, seed):
    """dict with cell_nodes (C x 8, caller numbering), coords, fracvol,
    density, pressure, velocity in the caller's numbering, and the maps
    cell_index / node_index (caller id -> structured id)."""
    rng = np.random.default_rng(seed)
    C, N = case.ncells, case.nnodes
    ci = rng.permutation(C)
    ni = rng.permutation(N)
    to_caller = np.empty(N, dtype=np.int64)
    to_caller[ni] = np.arange(N)
    cn = to_caller[structured_cell_nodes(case.nx, case.ny, case.nz)[ci]]
    return {"cell_nodes": cn, "coords": case.coords[ni], "fracvol": case.fracvol[:, ci],
            "density": case.density[:, ci], "pressure": case.pressure[:, ci], "velocity": case.velocity[ni],
            "cell_index": ci, "node_index": ni}
