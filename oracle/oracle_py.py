"""ctypes wrapper of the CPU restatement oracle (liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, as the checker.  The oracle takes the same
amcfd_params block the product's deck parser fills (include/amcfd.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DUMP = os.path.join(HERE, "_ref", "amcfd_ref_dump")
REF_CLI = os.path.join(HERE, "_ref", "AM-CFD")

_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle (plain C, FP64, no FMA contraction, like the reference build)."""
    src = os.path.join(HERE, "amcfd_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-std=c99", "-D_DEFAULT_SOURCE", "-ffp-contract=off",
                               "-fPIC", "-shared", src, "-o", LIB_PATH, "-lm"])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        VP = C.c_void_p
        L.orc_create.argtypes = [VP]
        L.orc_create.restype = VP
        L.orc_free.argtypes = [VP]
        L.orc_field.argtypes = [VP, C.c_char_p]
        L.orc_field.restype = C.POINTER(C.c_double)
        L.orc_dims.argtypes = [VP, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_step.argtypes = [VP, VP]
        L.orc_report.argtypes = [VP, VP]
        L.orc_get_state.argtypes = [VP, C.POINTER(C.c_double), C.POINTER(C.c_int)]
        for fn in ("orc_update_laser", "orc_meltpool", "orc_props", "orc_block_correct",
                   "orc_solve_entire", "orc_h2t", "orc_clean_velocities", "orc_correct_pressure",
                   "orc_fluxes", "orc_update_solutions", "orc_energy_assemble", "orc_outer_loop",
                   "orc_begin_step", "orc_species"):
            getattr(L, fn).argtypes = [VP]
        L.orc_free_surface.argtypes = [VP, C.POINTER(C.c_double)]
        for fn in ("orc_momentum", "orc_outer_iteration"):
            getattr(L, fn).argtypes = [VP]
            getattr(L, fn).restype = C.c_int
        for fn in ("orc_apply_bcs", "orc_discretize", "orc_source", "orc_residual",
                   "orc_solve_liquid"):
            getattr(L, fn).argtypes = [VP, C.c_int]
        _lib = L
    return _lib


class Oracle:
    """One oracle instance built from an amcfd_params block (ctypes Structure)."""

    def __init__(self, params):
        # params: an amcfd.Deck (kept alive: its tables back the pointers in the
        # parameter block) or an AmcfdParams whose owner outlives this call
        self._deck = params if hasattr(params, "params") else None
        params = params.params if self._deck is not None else params
        self._params = params
        self._h = C.c_void_p(lib().orc_create(C.byref(params)))
        ni, nj, nk = C.c_int(), C.c_int(), C.c_int()
        lib().orc_dims(self._h, C.byref(ni), C.byref(nj), C.byref(nk))
        self.ni, self.nj, self.nk = ni.value, nj.value, nk.value
        self.shape = (self.nk, self.nj, self.ni)

    def field(self, name: str) -> np.ndarray:
        """A live numpy view of an oracle array (3-D fields as [k][j][i])."""
        ptr = lib().orc_field(self._h, name.encode())
        if not ptr:
            raise KeyError(name)
        one_d = {"x": self.ni, "xu": self.ni, "dxpwinv": self.ni, "fracx": self.ni,
                 "y": self.nj, "yv": self.nj, "dypsinv": self.nj, "fracy": self.nj,
                 "z": self.nk, "zw": self.nk, "dzpbinv": self.nk, "fracz": self.nk,
                 "heatin": self.ni * self.nj, "areaij": self.ni * self.nj,
                 "areajk": self.nj * self.nk, "areaik": self.ni * self.nk, "fi": self.ni * self.nj}
        n = one_d.get(name, self.ni * self.nj * self.nk)
        arr = np.ctypeslib.as_array(ptr, shape=(n,))
        return arr if name in one_d else arr.reshape(self.shape)

    def step(self, report=None) -> Dict:
        from amcfd import AmcfdReport  # the report layout is the C ABI's
        r = report if report is not None else AmcfdReport()
        lib().orc_step(self._h, C.byref(r))
        return r.as_dict()

    def report(self) -> Dict:
        from amcfd import AmcfdReport
        r = AmcfdReport()
        lib().orc_report(self._h, C.byref(r))
        return r.as_dict()

    def free_surface(self) -> Dict:
        """FreeSurfaceManager::execute on the current state; its monitor values."""
        r = (C.c_double * 7)()
        lib().orc_free_surface(self._h, r)
        return {"lambda": r[0], "residual": r[1], "fi_min": r[2], "fi_max": r[3], "volume": r[4],
                "iterations": int(r[5]), "bracketed": int(r[6])}

    def box(self):
        t = C.c_double()
        b = (C.c_int * 7)()
        lib().orc_get_state(self._h, C.byref(t), b)
        return {"timet": t.value, "istat": b[0], "iend": b[1], "jstat": b[2], "jend": b[3],
                "kstat": b[4], "jstart": b[5], "istart": b[6]}

    def call(self, fn: str, *args):
        return getattr(lib(), "orc_" + fn)(self._h, *args)

    def close(self):
        if self._h:
            lib().orc_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
