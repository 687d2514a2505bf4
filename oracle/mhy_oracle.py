"""ctypes driver of the CPU oracle (mhy_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product.  Parity of the oracle with
the reference is unpinned (the reference has no golden data and cannot be built
without Arcane); see the header of mhy_oracle.cpp.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
_LIB = _HERE / "libmhy_oracle.so"

FIELD_IDS = {"density": 0, "internal_energy": 1, "pressure": 2, "sound_speed": 3,
             "pseudo_viscosity": 4, "cell_volume": 5, "cell_mass": 6, "caracteristic_length": 7,
             "velocity": 10, "node_mass": 11, "node_coord": 12, "env_mask": 50}


class _BC(ctypes.Structure):
    _fields_ = [("surface", ctypes.c_int), ("type", ctypes.c_int), ("value", ctypes.c_double)]


def build(force: bool = False) -> pathlib.Path:
    if force or not _LIB.exists() or _LIB.stat().st_mtime < (_HERE / "mhy_oracle.cpp").stat().st_mtime:
        subprocess.run(["make", "-C", str(_HERE), "-s"], check=True)
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(_LIB))
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int] * 3 + [dp, ctypes.c_int, dp] + [ctypes.c_double] * 6 + \
            [ctypes.c_int] * 5 + [ctypes.POINTER(_BC), ctypes.c_int, ctypes.POINTER(ctypes.c_int), dp] + [ctypes.c_int] * 6
        L.orc_init.argtypes = [ctypes.c_void_p, dp, dp, dp, dp]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_scalars.argtypes = [ctypes.c_void_p, dp]
        L.orc_get_field.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.orc_get_field.restype = ctypes.c_int
        L.orc_pow_third.argtypes = [ctypes.c_double, ctypes.c_int]
        L.orc_pow_third.restype = ctypes.c_double
        L.orc_set_option.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
        L.orc_set_option.restype = ctypes.c_int
        L.orc_set_dt_reduction.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 3
        L.orc_set_dt_reduction.restype = ctypes.c_int
        L.orc_dt_local_min.argtypes = [ctypes.c_void_p]
        L.orc_dt_local_min.restype = ctypes.c_double
        L.orc_dt_finish.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.orc_halo_count.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_halo_count.restype = ctypes.c_long
        for name in ("orc_halo_pack", "orc_halo_unpack"):
            getattr(L, name).argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 4 + [dp]
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def pow_third(v: float, project: bool = True) -> float:
    """V^(1./3.) as the oracle computes it (project cube root or std::pow)."""
    return lib().orc_pow_third(float(v), 1 if project else 0)


class Oracle:
    """One problem instance on the CPU oracle.

    pow_mode: "project" evaluates V^(1/3.) with the shared project cube root
    (bitwise comparable with the GPU); "libm" uses std::pow as the reference does
    on a CPU (differs from "project" by 1 ulp in ~0.1% of evaluations)."""

    def __init__(self, case, pow_mode: str = "project", threads: int | None = None):
        L = lib()
        if threads is not None:
            L.orc_set_threads(int(threads))
        o = case.options
        self.case = case
        coords = np.ascontiguousarray(case.coords, dtype=np.float64)
        gam = np.ascontiguousarray(case.gamma, dtype=np.float64)
        bcs = (_BC * max(1, len(o.boundary_conditions)))(*[_BC(s, t, v) for s, t, v in o.boundary_conditions])
        eos = np.zeros(case.nenv, dtype=np.int32)
        pinf = np.full(case.nenv, 0.01)                 # StiffenedGasEOS.axl:104 default
        for k, kind in enumerate(getattr(o, "eos", ()) or ()):
            eos[k] = kind
        for k, v in enumerate(getattr(o, "limit_tension", ()) or ()):
            pinf[k] = v
        self._keep = (coords, gam, bcs, eos, pinf)
        self.h = L.orc_create(case.nx, case.ny, case.nz, _dp(coords), case.nenv, _dp(gam),
                              o.cfl, o.threshold, o.deltat_init, o.deltat_min, o.deltat_max, o.final_time,
                              o.longueur_caracteristique, o.pseudo_centree, o.ordre_projection,
                              o.projection_limiteur_id, len(o.boundary_conditions), bcs,
                              1 if pow_mode == "project" else 0,
                              eos.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(pinf),
                              int(getattr(o, "with_newton", 0)), int(getattr(o, "schema_csts", 0)),
                              int(getattr(o, "pente_borne", 0)), int(getattr(o, "pente_borne_debar_fix", 0)),
                              int(getattr(o, "pente_borne_mixte", 0)), int(getattr(o, "limiteur_pure_id", 0)))
        if int(getattr(o, "conservation_energie_totale", 0)):
            if L.orc_set_option(self.h, b"conservation_energie_totale", 1) != 0:
                raise RuntimeError("oracle: unknown option")
        fv = np.ascontiguousarray(case.fracvol, dtype=np.float64)
        de = np.ascontiguousarray(case.density, dtype=np.float64)
        pr = np.ascontiguousarray(case.pressure, dtype=np.float64)
        ve = np.ascontiguousarray(case.velocity, dtype=np.float64)
        L.orc_init(self.h, _dp(fv), _dp(de), _dp(pr), _dp(ve))

    def step(self, ncycles: int = 1):
        lib().orc_step(self.h, int(ncycles))

    def scalars(self) -> dict:
        out = np.zeros(6)
        lib().orc_get_scalars(self.h, _dp(out))
        return {"dt": out[0], "old_dt": out[1], "time": out[2], "sens": int(out[3]),
                "iteration": int(out[4]), "status": int(out[5])}

    def field(self, name: str) -> np.ndarray:
        c = self.case
        if name in ("velocity", "node_coord"):
            out = np.zeros((c.nnodes, 3))
        elif name == "node_mass":
            out = np.zeros(c.nnodes)
        else:
            out = np.zeros(c.ncells)
        rc = lib().orc_get_field(self.h, FIELD_IDS[name], _dp(out))
        if rc != 0:
            raise KeyError(name)
        return out

    def env_field(self, which: str, k: int) -> np.ndarray:
        base = {"fracvol": 20, "density": 30, "internal_energy": 40}[which]
        out = np.zeros(self.case.ncells)
        if lib().orc_get_field(self.h, base + k, _dp(out)) != 0:
            raise KeyError(which)
        return out

    def env_mask(self) -> np.ndarray:
        out = np.zeros(self.case.ncells)
        if lib().orc_get_field(self.h, 50, _dp(out)) != 0:
            raise KeyError("env_mask")
        return out.astype(np.uint32)

    # slabs (one environment): dt over owned cell layers, combined outside
    def set_dt_reduction(self, k_lo: int, k_hi: int, external: bool = True):
        if lib().orc_set_dt_reduction(self.h, int(k_lo), int(k_hi), int(external)) != 0:
            raise ValueError("bad dt layer range")

    def dt_local_min(self) -> float:
        return lib().orc_dt_local_min(self.h)

    def dt_finish(self, minimum: float):
        lib().orc_dt_finish(self.h, float(minimum))

    def halo_count(self, cell_layers: int, node_layers: int) -> int:
        return int(lib().orc_halo_count(self.h, int(cell_layers), int(node_layers)))

    def halo_pack(self, clo, chi, nlo, nhi) -> np.ndarray:
        out = np.empty(self.halo_count(chi - clo, nhi - nlo))
        if lib().orc_halo_pack(self.h, clo, chi, nlo, nhi, _dp(out)) != 0:
            raise ValueError("bad layer range")
        return out

    def halo_unpack(self, clo, chi, nlo, nhi, buf: np.ndarray):
        buf = np.ascontiguousarray(buf, dtype=np.float64)
        if buf.size != self.halo_count(chi - clo, nhi - nlo) or lib().orc_halo_unpack(self.h, clo, chi, nlo, nhi, _dp(buf)) != 0:
            raise ValueError("bad layer range or buffer")

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run(case, cycles=None, pow_mode="project", threads=None, record_dt=False):
    """Run `cycles` cycles; return (oracle, dt list if record_dt)."""
    o = Oracle(case, pow_mode=pow_mode, threads=threads)
    n = case.cycles if cycles is None else cycles
    dts = []
    if record_dt:
        for _ in range(n):
            dts.append(o.scalars()["dt"])
            o.step(1)
    else:
        o.step(n)
    return o, dts


if __name__ == "__main__":  # quick manual check
    import sys
    sys.path.insert(0, str(_HERE.parent / "arcane-benchs_b200"))
    from mhy_b200 import gen
    c = gen.sod()
    o, dts = run(c, 200, record_dt=True)
    print(o.scalars(), dts[:3], dts[-1])
    print(o.field("density")[::5][:20])
