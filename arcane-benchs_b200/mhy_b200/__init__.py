"""ctypes binding of the C ABI in include/mhy.h (libmhy_b200.so, sm_100a).

There is no CPU fallback: loading fails with an exception when the CUDA
library has not been built or no GPU is present.
"""
from __future__ import annotations

import ctypes
import pathlib

import numpy as np

from . import gen  # noqa: F401  (re-export)

_PKG = pathlib.Path(__file__).resolve().parent.parent
LIB_PATH = _PKG / "lib" / "libmhy_b200.so"

MHY_MAX_BC = 16
MHY_MAX_ENV = 8

FIELDS = {"density": 0, "internal_energy": 1, "pressure": 2, "sound_speed": 3, "pseudo_viscosity": 4,
          "cell_volume": 5, "cell_mass": 6, "caracteristic_length": 7, "velocity": 10, "node_mass": 11,
          "node_coord": 12}
STATUS_DT_MIN, STATUS_FINAL_TIME, STATUS_NAN_DT, STATUS_ZERO_MASS = 1, 2, 4, 8
ERRORS = {-1: "MHY_ERR_ARG", -2: "MHY_ERR_CUDA", -3: "MHY_ERR_OOM", -4: "MHY_ERR_UNSUPPORTED",
          -5: "MHY_ERR_ORDER", -6: "MHY_ERR_DT_MIN", -7: "MHY_ERR_NUMERIC", -8: "MHY_ERR_STATE"}

# every symbol include/mhy.h declares
EXPORTED = ["mhy_options_default", "mhy_create", "mhy_set_state", "mhy_hydro_start_init",
            "mhy_save_values_at_n", "mhy_update_velocity", "mhy_apply_boundary_condition",
            "mhy_update_position", "mhy_compute_geometric_values", "mhy_update_density",
            "mhy_compute_artificial_viscosity", "mhy_update_energy_and_pressure", "mhy_remap",
            "mhy_compute_delta_t", "mhy_step", "mhy_synchronize", "mhy_get_field", "mhy_get_dt",
            "mhy_get_time", "mhy_get_status", "mhy_get_sizes", "mhy_get_stream", "mhy_kernels_per_cycle",
            "mhy_last_error", "mhy_destroy", "mhy_compute_hydro_dt_noalloc", "mhy_get_env_field",
            "mhy_get_env_mask", "mhy_batch_create", "mhy_batch_set_state", "mhy_batch_hydro_start_init",
            "mhy_batch_step", "mhy_batch_synchronize", "mhy_batch_get_field", "mhy_batch_get_dt",
            "mhy_batch_get_status", "mhy_batch_size", "mhy_batch_kernels_per_cycle", "mhy_batch_get_stream",
            "mhy_batch_destroy", "mhy_checkpoint_size", "mhy_checkpoint_save", "mhy_checkpoint_load",
            "mhy_get_totals", "mhy_batch_get_totals", "mhy_autotune", "mhy_set_tuning", "mhy_get_tuning",
            "mhy_batch_autotune", "mhy_batch_set_tuning", "mhy_batch_get_tuning", "mhy_create_csr",
            "mhy_csr_structure", "mhy_set_dt_reduction", "mhy_dt_local_min", "mhy_dt_finish", "mhy_halo_bytes",
            "mhy_halo_pack", "mhy_halo_unpack"]
MHY_TUNE_SLOTS = 10
TUNE_SLOTS = ("lagrange_nodes", "lagrange_cells", "cells_x", "cells_y", "cells_z", "nodes_x", "nodes_y", "nodes_z",
              "dt_min", "dt_finish")
ENV_FIELDS = {"fracvol": 0, "density": 1, "internal_energy": 2, "pressure": 3, "sound_speed": 4,
              "mass_fraction": 5, "cell_mass": 6}


class MhyError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class BC(ctypes.Structure):
    _fields_ = [("surface", ctypes.c_int32), ("type", ctypes.c_int32), ("value", ctypes.c_double)]


class CTuning(ctypes.Structure):
    """mhy_tuning: per kernel slot (TUNE_SLOTS) the work order and grid
    percentage (batches) and the lines per block of the y/z sweeps."""
    _fields_ = [("order", ctypes.c_int32 * MHY_TUNE_SLOTS), ("occupancy_pct", ctypes.c_int32 * MHY_TUNE_SLOTS),
                ("lines_per_block", ctypes.c_int32 * MHY_TUNE_SLOTS),
                ("ms_default", ctypes.c_double * MHY_TUNE_SLOTS), ("ms_tuned", ctypes.c_double * MHY_TUNE_SLOTS),
                ("from_cache", ctypes.c_int32), ("trials", ctypes.c_int32)]

    @classmethod
    def default(cls) -> "CTuning":
        t = cls()
        for k in range(MHY_TUNE_SLOTS):
            t.order[k], t.occupancy_pct[k], t.lines_per_block[k] = 0, 100, 8
        return t

    def as_dict(self) -> dict:
        return {"slots": {name: {"order": self.order[k], "occupancy_pct": self.occupancy_pct[k],
                                 "lines_per_block": self.lines_per_block[k],
                                 "ms_default": round(self.ms_default[k], 4), "ms_tuned": round(self.ms_tuned[k], 4)}
                          for k, name in enumerate(TUNE_SLOTS)},
                "from_cache": bool(self.from_cache), "trials": self.trials}


class COptions(ctypes.Structure):
    _fields_ = [("cfl", ctypes.c_double), ("threshold", ctypes.c_double), ("deltat_init", ctypes.c_double),
                ("deltat_min", ctypes.c_double), ("deltat_max", ctypes.c_double), ("final_time", ctypes.c_double),
                ("longueur_caracteristique", ctypes.c_int32), ("pseudo_centree", ctypes.c_int32),
                ("ordre_projection", ctypes.c_int32), ("projection_limiteur_id", ctypes.c_int32),
                ("nb_bc", ctypes.c_int32), ("bc", BC * MHY_MAX_BC), ("nb_env", ctypes.c_int32),
                ("adiabatic_cst", ctypes.c_double * MHY_MAX_ENV), ("precision", ctypes.c_int32),
                ("eos", ctypes.c_int32 * MHY_MAX_ENV), ("limit_tension", ctypes.c_double * MHY_MAX_ENV),
                ("with_newton", ctypes.c_int32), ("schema_csts", ctypes.c_int32),
                ("projection_pente_borne", ctypes.c_int32), ("pente_borne_debar_fix", ctypes.c_int32),
                ("pente_borne_mixte", ctypes.c_int32), ("limiteur_pure_id", ctypes.c_int32),
                ("conservation_energie_totale", ctypes.c_int32)]


class CMesh(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("node_coords", ctypes.POINTER(ctypes.c_double))]


class CCsrMesh(ctypes.Structure):
    _fields_ = [("ncells", ctypes.c_int64), ("nnodes", ctypes.c_int64),
                ("cell_node_offsets", ctypes.POINTER(ctypes.c_int64)), ("cell_nodes", ctypes.POINTER(ctypes.c_int64)),
                ("node_coords", ctypes.POINTER(ctypes.c_double))]


class CState(ctypes.Structure):
    _fields_ = [("fracvol", ctypes.POINTER(ctypes.c_double)), ("density", ctypes.POINTER(ctypes.c_double)),
                ("pressure", ctypes.POINTER(ctypes.c_double)), ("velocity", ctypes.POINTER(ctypes.c_double))]


_lib = None


def load(path: pathlib.Path | str | None = None):
    """Load the shared library (no GPU call is made)."""
    global _lib
    if _lib is not None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with arcane-benchs_b200/build.py (no CPU fallback exists)")
    L = ctypes.CDLL(str(p))
    vp = ctypes.c_void_p
    L.mhy_options_default.argtypes = [ctypes.POINTER(COptions)]
    L.mhy_options_default.restype = None
    L.mhy_create.argtypes = [ctypes.POINTER(CMesh), ctypes.POINTER(COptions), ctypes.c_int, ctypes.POINTER(vp)]
    L.mhy_set_state.argtypes = [vp, ctypes.POINTER(CState)]
    for name in ["mhy_hydro_start_init", "mhy_save_values_at_n", "mhy_update_velocity",
                 "mhy_apply_boundary_condition", "mhy_update_position", "mhy_compute_geometric_values",
                 "mhy_update_density", "mhy_compute_artificial_viscosity", "mhy_update_energy_and_pressure",
                 "mhy_remap", "mhy_compute_delta_t", "mhy_synchronize", "mhy_kernels_per_cycle"]:
        getattr(L, name).argtypes = [vp]
        getattr(L, name).restype = ctypes.c_int
    L.mhy_step.argtypes = [vp, ctypes.c_int]
    L.mhy_get_field.argtypes = [vp, ctypes.c_int, vp, ctypes.c_size_t]
    L.mhy_get_dt.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.mhy_get_time.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
    L.mhy_get_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32)]
    L.mhy_get_sizes.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int64)] * 3
    L.mhy_get_stream.argtypes = [vp]
    L.mhy_get_stream.restype = vp
    L.mhy_last_error.restype = ctypes.c_char_p
    L.mhy_destroy.argtypes = [vp]
    L.mhy_destroy.restype = None
    L.mhy_compute_hydro_dt_noalloc.argtypes = [ctypes.c_int32] * 3 + [vp] * 3 + [ctypes.c_double] * 3 + [vp, vp]
    L.mhy_compute_hydro_dt_noalloc.restype = ctypes.c_int
    L.mhy_get_env_field.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_size_t]
    L.mhy_get_env_mask.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.c_size_t]
    L.mhy_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(CMesh), ctypes.POINTER(COptions), ctypes.c_int,
                                   ctypes.POINTER(vp)]
    L.mhy_batch_set_state.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CState)]
    for name in ["mhy_batch_hydro_start_init", "mhy_batch_synchronize", "mhy_batch_size",
                 "mhy_batch_kernels_per_cycle"]:
        getattr(L, name).argtypes = [vp]
        getattr(L, name).restype = ctypes.c_int
    L.mhy_batch_step.argtypes = [vp, ctypes.c_int]
    L.mhy_batch_get_field.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_size_t]
    L.mhy_batch_get_dt.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.mhy_batch_get_status.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_uint32)]
    L.mhy_batch_get_stream.argtypes = [vp]
    L.mhy_batch_get_stream.restype = vp
    L.mhy_batch_destroy.argtypes = [vp]
    L.mhy_batch_destroy.restype = None
    L.mhy_get_totals.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.mhy_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CTuning)]
    L.mhy_set_tuning.argtypes = [vp, ctypes.POINTER(CTuning)]
    L.mhy_get_tuning.argtypes = [vp, ctypes.POINTER(CTuning)]
    L.mhy_batch_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(CTuning)]
    L.mhy_batch_set_tuning.argtypes = [vp, ctypes.POINTER(CTuning)]
    L.mhy_batch_get_tuning.argtypes = [vp, ctypes.POINTER(CTuning)]
    L.mhy_batch_get_totals.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.mhy_checkpoint_size.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t)]
    L.mhy_checkpoint_save.argtypes = [vp, vp, ctypes.c_size_t]
    L.mhy_checkpoint_load.argtypes = [vp, vp, ctypes.c_size_t]
    i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
    L.mhy_csr_structure.argtypes = [ctypes.c_int64, ctypes.c_int64, i64p, i64p, i32p, i32p, i32p]
    L.mhy_csr_structure.restype = ctypes.c_int
    L.mhy_create_csr.argtypes = [ctypes.POINTER(CCsrMesh), ctypes.POINTER(COptions), ctypes.c_int, ctypes.POINTER(vp)]
    L.mhy_create_csr.restype = ctypes.c_int
    L.mhy_set_dt_reduction.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
    L.mhy_dt_local_min.argtypes = [vp, vp]
    L.mhy_dt_finish.argtypes = [vp, vp]
    L.mhy_halo_bytes.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_size_t)]
    L.mhy_halo_pack.argtypes = [vp] + [ctypes.c_int32] * 4 + [vp, ctypes.c_size_t]
    L.mhy_halo_unpack.argtypes = [vp] + [ctypes.c_int32] * 4 + [vp, ctypes.c_size_t]
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise MhyError(rc, load().mhy_last_error().decode())
    return rc


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def csr_structure(cell_nodes: np.ndarray, nnodes: int):
    """mhy_csr_structure: (dims, cell_index, node_index) of a logically
    Cartesian hexahedral block given as cell -> node connectivity
    (ncells x 8, SN_trigo local order, any numbering).  Host only."""
    cn = np.ascontiguousarray(cell_nodes, dtype=np.int64).reshape(-1)
    ncells = cn.size // 8
    off = np.arange(0, 8 * ncells + 1, 8, dtype=np.int64)
    dims = np.zeros(3, dtype=np.int32)
    ci = np.zeros(ncells, dtype=np.int32)
    ni = np.zeros(int(nnodes), dtype=np.int32)
    i32 = ctypes.POINTER(ctypes.c_int32)
    i64 = ctypes.POINTER(ctypes.c_int64)
    _check(load().mhy_csr_structure(ncells, int(nnodes), off.ctypes.data_as(i64), cn.ctypes.data_as(i64),
                                    dims.ctypes.data_as(i32), ci.ctypes.data_as(i32), ni.ctypes.data_as(i32)))
    return tuple(int(d) for d in dims), ci, ni


def make_options(opts, gammas) -> COptions:
    o = COptions()
    load().mhy_options_default(ctypes.byref(o))
    o.cfl, o.threshold = opts.cfl, opts.threshold
    o.deltat_init, o.deltat_min, o.deltat_max = opts.deltat_init, opts.deltat_min, opts.deltat_max
    o.final_time = opts.final_time
    o.longueur_caracteristique = opts.longueur_caracteristique
    o.pseudo_centree = opts.pseudo_centree
    o.ordre_projection = opts.ordre_projection
    o.projection_limiteur_id = opts.projection_limiteur_id
    o.nb_bc = len(opts.boundary_conditions)
    for b, (s, t, v) in enumerate(opts.boundary_conditions):
        o.bc[b] = BC(s, t, v)
    o.precision = int(getattr(opts, "precision", 0))
    o.nb_env = len(gammas)
    for k, g in enumerate(gammas):
        o.adiabatic_cst[k] = float(g)
    o.with_newton = int(getattr(opts, "with_newton", 0))
    o.schema_csts = int(getattr(opts, "schema_csts", 0))
    o.projection_pente_borne = int(getattr(opts, "pente_borne", 0))
    o.pente_borne_debar_fix = int(getattr(opts, "pente_borne_debar_fix", 0))
    o.pente_borne_mixte = int(getattr(opts, "pente_borne_mixte", 0))
    o.limiteur_pure_id = int(getattr(opts, "limiteur_pure_id", 0))
    o.conservation_energie_totale = int(getattr(opts, "conservation_energie_totale", 0))
    for k, kind in enumerate(getattr(opts, "eos", ()) or ()):
        o.eos[k] = int(kind)
    for k, v in enumerate(getattr(opts, "limit_tension", ()) or ()):
        o.limit_tension[k] = float(v)
    return o


class Context:
    """One mesh instance on one GPU (mhy_ctx)."""

    def __init__(self, case, device: int = -1, init: bool = True):
        L = load()
        self.case = case
        self._coords = np.ascontiguousarray(case.coords, dtype=np.float64)
        mesh = CMesh(case.nx, case.ny, case.nz, _dp(self._coords))
        opt = make_options(case.options, case.gamma)
        h = ctypes.c_void_p()
        _check(L.mhy_create(ctypes.byref(mesh), ctypes.byref(opt), device, ctypes.byref(h)))
        self.h = h
        fv = np.ascontiguousarray(case.fracvol, dtype=np.float64)
        de = np.ascontiguousarray(case.density, dtype=np.float64)
        pr = np.ascontiguousarray(case.pressure, dtype=np.float64)
        ve = np.ascontiguousarray(case.velocity, dtype=np.float64)
        st = CState(_dp(fv), _dp(de), _dp(pr), _dp(ve))
        _check(L.mhy_set_state(self.h, ctypes.byref(st)))
        if init:
            _check(L.mhy_hydro_start_init(self.h))

    # the compute-loop entry points in the reference order
    def cycle_by_entry_points(self):
        L = load()
        for name in ["mhy_save_values_at_n", "mhy_update_velocity", "mhy_apply_boundary_condition",
                     "mhy_update_position", "mhy_compute_geometric_values", "mhy_update_density",
                     "mhy_compute_artificial_viscosity", "mhy_update_energy_and_pressure", "mhy_remap",
                     "mhy_compute_delta_t"]:
            _check(getattr(L, name)(self.h))

    def step(self, ncycles: int = 1):
        _check(load().mhy_step(self.h, int(ncycles)))

    def synchronize(self):
        _check(load().mhy_synchronize(self.h))

    def dt(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(load().mhy_get_dt(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def time(self):
        t, it = ctypes.c_double(), ctypes.c_int64()
        _check(load().mhy_get_time(self.h, ctypes.byref(t), ctypes.byref(it)))
        return t.value, it.value

    def status(self) -> int:
        f = ctypes.c_uint32()
        _check(load().mhy_get_status(self.h, ctypes.byref(f)))
        return f.value

    def autotune(self, cycles: int = 2) -> CTuning:
        """mhy_autotune: lines per block of the y/z sweeps, timed on this
        context's state (restored afterwards)."""
        t = CTuning()
        _check(load().mhy_autotune(self.h, int(cycles), ctypes.byref(t)))
        return t

    def tuning(self) -> CTuning:
        t = CTuning()
        _check(load().mhy_get_tuning(self.h, ctypes.byref(t)))
        return t

    def set_tuning(self, t: CTuning):
        _check(load().mhy_set_tuning(self.h, ctypes.byref(t)))

    def totals(self) -> dict:
        """Compensated device sums: mass, internal, kinetic and total energy."""
        out = (ctypes.c_double * 3)()
        _check(load().mhy_get_totals(self.h, out))
        return {"mass": out[0], "internal_energy": out[1], "kinetic_energy": out[2],
                "total_energy": out[1] + out[2]}

    def kernels_per_cycle(self) -> int:
        return load().mhy_kernels_per_cycle(self.h)

    def stream(self) -> int:
        return load().mhy_get_stream(self.h) or 0

    def field(self, name: str) -> np.ndarray:
        c = self.case
        fid = FIELDS[name]
        if name in ("velocity", "node_coord"):
            out = np.empty((c.nnodes, 3))
        elif name == "node_mass":
            out = np.empty(c.nnodes)
        else:
            out = np.empty(c.ncells)
        _check(load().mhy_get_field(self.h, fid, out.ctypes.data_as(ctypes.c_void_p), out.nbytes))
        return out

    def save_checkpoint(self) -> bytes:
        """Restart dump of the state between cycles (mhy_checkpoint_save)."""
        L = load()
        n = ctypes.c_size_t()
        _check(L.mhy_checkpoint_size(self.h, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _check(L.mhy_checkpoint_save(self.h, buf, n.value))
        return buf.raw

    @classmethod
    def from_csr(cls, case, cell_nodes, node_coords, fracvol, density, pressure, velocity, device: int = -1):
        """mhy_create_csr: a context on explicit connectivity in the caller's
        numbering (cell_nodes: ncells x 8 node ids, SN_trigo order), with the
        initial state in the same numbering; case gives the options and gases.
        Fields come back in the caller's numbering."""
        self = cls.__new__(cls)
        L = load()
        self.case = case
        cn = np.ascontiguousarray(cell_nodes, dtype=np.int64).reshape(-1)
        off = np.arange(0, cn.size + 1, 8, dtype=np.int64)
        self._coords = np.ascontiguousarray(node_coords, dtype=np.float64)
        i64 = ctypes.POINTER(ctypes.c_int64)
        mesh = CCsrMesh(cn.size // 8, self._coords.shape[0], off.ctypes.data_as(i64), cn.ctypes.data_as(i64),
                        _dp(self._coords))
        opt = make_options(case.options, case.gamma)
        h = ctypes.c_void_p()
        _check(L.mhy_create_csr(ctypes.byref(mesh), ctypes.byref(opt), device, ctypes.byref(h)))
        self.h = h
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (fracvol, density, pressure, velocity)]
        st = CState(*[_dp(a) for a in arrs])
        _check(L.mhy_set_state(self.h, ctypes.byref(st)))
        _check(L.mhy_hydro_start_init(self.h))
        return self

    @classmethod
    def from_checkpoint(cls, case, blob: bytes, device: int = -1):
        """A context on case's mesh and options, resumed from a restart dump."""
        self = cls.__new__(cls)
        L = load()
        self.case = case
        self._coords = np.ascontiguousarray(case.coords, dtype=np.float64)
        mesh = CMesh(case.nx, case.ny, case.nz, _dp(self._coords))
        opt = make_options(case.options, case.gamma)
        h = ctypes.c_void_p()
        _check(L.mhy_create(ctypes.byref(mesh), ctypes.byref(opt), device, ctypes.byref(h)))
        self.h = h
        buf = ctypes.create_string_buffer(blob, len(blob))
        _check(L.mhy_checkpoint_load(self.h, buf, len(blob)))
        return self

    def env_field(self, name: str, k: int) -> np.ndarray:
        """Value of environment k in every cell (0 where the cell does not hold it)."""
        out = np.empty(self.case.ncells)
        _check(load().mhy_get_env_field(self.h, ENV_FIELDS[name], int(k), out.ctypes.data_as(ctypes.c_void_p),
                                        out.nbytes))
        return out

    # slabs: dt over owned cell layers, combined and finished by the caller;
    # the ghost layers' state moved through device buffers (data pointers)
    def set_dt_reduction(self, k_lo: int, k_hi: int, external: bool = True):
        _check(load().mhy_set_dt_reduction(self.h, int(k_lo), int(k_hi), int(external)))

    def dt_local_min(self, dev_ptr: int):
        _check(load().mhy_dt_local_min(self.h, ctypes.c_void_p(dev_ptr)))

    def dt_finish(self, dev_ptr: int):
        _check(load().mhy_dt_finish(self.h, ctypes.c_void_p(dev_ptr)))

    def halo_bytes(self, cell_layers: int, node_layers: int) -> int:
        n = ctypes.c_size_t()
        _check(load().mhy_halo_bytes(self.h, int(cell_layers), int(node_layers), ctypes.byref(n)))
        return n.value

    def halo_pack(self, clo, chi, nlo, nhi, dev_ptr: int, nbytes: int):
        _check(load().mhy_halo_pack(self.h, clo, chi, nlo, nhi, ctypes.c_void_p(dev_ptr), nbytes))

    def halo_unpack(self, clo, chi, nlo, nhi, dev_ptr: int, nbytes: int):
        _check(load().mhy_halo_unpack(self.h, clo, chi, nlo, nhi, ctypes.c_void_p(dev_ptr), nbytes))

    def env_mask(self) -> np.ndarray:
        out = np.empty(self.case.ncells, dtype=np.uint32)
        _check(load().mhy_get_env_mask(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), out.nbytes))
        return out

    def close(self):
        if getattr(self, "h", None):
            load().mhy_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent meshes advanced together on one GPU (mhy_batch); every
    instance has the same number of environments."""

    def __init__(self, cases, device: int = -1, init: bool = True):
        L = load()
        self.cases = list(cases)
        n = len(self.cases)
        self._keep = []
        meshes = (CMesh * n)()
        opts = (COptions * n)()
        for i, c in enumerate(self.cases):
            xyz = np.ascontiguousarray(c.coords, dtype=np.float64)
            self._keep.append(xyz)
            meshes[i] = CMesh(c.nx, c.ny, c.nz, _dp(xyz))
            opts[i] = make_options(c.options, c.gamma)
        h = ctypes.c_void_p()
        _check(L.mhy_batch_create(n, meshes, opts, device, ctypes.byref(h)))
        self.h = h
        for i, c in enumerate(self.cases):
            arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (c.fracvol, c.density, c.pressure, c.velocity)]
            st = CState(*[_dp(a) for a in arrs])
            _check(L.mhy_batch_set_state(self.h, i, ctypes.byref(st)))
        if init:
            _check(L.mhy_batch_hydro_start_init(self.h))

    def step(self, ncycles: int = 1):
        _check(load().mhy_batch_step(self.h, int(ncycles)))

    def size(self) -> int:
        return load().mhy_batch_size(self.h)

    def synchronize(self):
        _check(load().mhy_batch_synchronize(self.h))

    def dt(self, i: int):
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(load().mhy_batch_get_dt(self.h, int(i), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def status(self, i: int) -> int:
        f = ctypes.c_uint32()
        _check(load().mhy_batch_get_status(self.h, int(i), ctypes.byref(f)))
        return f.value

    def autotune(self, cycles: int = 2) -> CTuning:
        """mhy_batch_autotune: the fastest work order, persistent grid and
        lines per block per kernel slot, timed on this batch's state (restored
        afterwards)."""
        t = CTuning()
        _check(load().mhy_batch_autotune(self.h, int(cycles), ctypes.byref(t)))
        return t

    def tuning(self) -> CTuning:
        t = CTuning()
        _check(load().mhy_batch_get_tuning(self.h, ctypes.byref(t)))
        return t

    def set_tuning(self, t: CTuning):
        _check(load().mhy_batch_set_tuning(self.h, ctypes.byref(t)))

    def totals(self, i: int) -> dict:
        out = (ctypes.c_double * 3)()
        _check(load().mhy_batch_get_totals(self.h, int(i), out))
        return {"mass": out[0], "internal_energy": out[1], "kinetic_energy": out[2],
                "total_energy": out[1] + out[2]}

    def kernels_per_cycle(self) -> int:
        return load().mhy_batch_kernels_per_cycle(self.h)

    def stream(self) -> int:
        return load().mhy_batch_get_stream(self.h) or 0

    def field(self, i: int, name: str) -> np.ndarray:
        c = self.cases[i]
        if name in ("velocity", "node_coord"):
            out = np.empty((c.nnodes, 3))
        elif name == "node_mass":
            out = np.empty(c.nnodes)
        else:
            out = np.empty(c.ncells)
        _check(load().mhy_batch_get_field(self.h, int(i), FIELDS[name], out.ctypes.data_as(ctypes.c_void_p),
                                          out.nbytes))
        return out

    def close(self):
        if getattr(self, "h", None):
            load().mhy_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
