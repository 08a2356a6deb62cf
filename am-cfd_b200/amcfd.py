"""Python binding of the B200 melt-pool solver's C ABI (include/amcfd.h).

This is the host-side mirror of the reference's in-process interface
(CFDSolverManager.h:96-104 driven by src/main.cpp:123-201): a deck is parsed,
a solver context is created on one GPU, and each call to ``Solver.step()``
performs one time step (timet += delt, updateLaser, iterativeLoopSolve,
updateSolutions) on the device.  Fields are read back by the reference's
registry keys ("temp", "uvel", ...).

The binding loads ``libamcfd_b200.so`` built in this directory; there is no
fallback: a missing library is an error.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libamcfd_b200.so")
MAX_ZONES = 32

SCHEME_UPWIND, SCHEME_POWER_LAW, SCHEME_EXPONENTIAL = 0, 1, 2
ORDER_EXACT, ORDER_REDBLACK = 0, 1
PREC_FP64, PREC_FP32, PREC_FP32_DC = 0, 1, 2
WS_OFF, WS_PREDICT, WS_RECORD, WS_PREDICT_H = 0, 1, 2, 3
PHASES = {"laser": 1, "energy_assemble": 2, "energy_solve": 3, "h2t": 4, "meltpool": 5,
          "momentum": 6, "converge": 7, "update": 8, "species": 9}
ERRORS = {0: "AMCFD_OK", -1: "AMCFD_E_ARG", -2: "AMCFD_E_IO", -3: "AMCFD_E_PARSE",
          -4: "AMCFD_E_CUDA", -5: "AMCFD_E_NONFINITE", -6: "AMCFD_E_TIMEOUT",
          -7: "AMCFD_E_NOMEM", -8: "AMCFD_E_CAPACITY"}

_D = C.c_double
_I = C.c_int


class AmcfdParams(C.Structure):
    _fields_ = [("nzx", _I), ("nzy", _I), ("nzz", _I),
                ("xzone", _D * MAX_ZONES), ("ncvx", _D * MAX_ZONES), ("powrx", _D * MAX_ZONES),
                ("yzone", _D * MAX_ZONES), ("ncvy", _D * MAX_ZONES), ("powry", _D * MAX_ZONES),
                ("zzone", _D * MAX_ZONES), ("ncvz", _D * MAX_ZONES), ("powrz", _D * MAX_ZONES)] + \
        [(n, _D) for n in ("dens denl viscos tsolid tliquid hsmelt hlfriz acpa acpb acpl "
                           "thconsa thconsb thconsc thconla thconlb urfu urfv urfw urfp urfh "
                           "htci htcj htck1 htckn emiss tempwest tempeast tempnorth tempbottom "
                           "temppreheat beta dgdtp darcyKo a_oxygen grav sigm tempamb pressamb "
                           "gasconst alaspow alaseta alasrb alasfact lasertime xstart ystart "
                           "scanvel avolpow apowseta heatthick heatrb avolfact").split()] + \
        [("isevap", _I)] + [(n, _D) for n in "evaplatent evaptemp evapfact molarmass".split()] + \
        [(n, _D) for n in "delt outtime finaltime nonlintol".split()] + \
        [(n, _I) for n in "maxit scheme navierstokes steady udtoolpath ntool".split()] + \
        [("tool_txyz", C.POINTER(_D)), ("tool_on", C.POINTER(_I)), ("tool_id", C.POINTER(_I)),
         ("nheattable", _I), ("heattable", C.POINTER(_D)),
         ("nvardt", _I), ("vardt", C.POINTER(_D))] + \
        [(n, _I) for n in "powderbed movingmesh species freesurface".split()] + \
        [(n, _D) for n in "initconc massdiff kp urfc".split()] + \
        [(n, _I) for n in "numlayers ncvzlayer".split()] + \
        [(n, _D) for n in "layerheight powderden powdercpa powdercpb powderthcona powderthconb".split()] + \
        [(n, _I) for n in "xmoveindex ymoveindex solidification".split()] + \
        [(n, _D) for n in ("fs_lam1 fs_lam2 fs_surftens fs_maxiterenergy fs_tolenergy fs_maxiterbisect "
                           "fs_tolbisect fs_urfree").split()]


class AmcfdFreeSurface(C.Structure):
    _fields_ = [(n, _D) for n in "lambda residual fi_min fi_max volume".split()] + \
        [("iterations", _I), ("bracketed", _I)]


class AmcfdReport(C.Structure):
    _fields_ = [("timet", _D), ("niter", _I), ("itertot", _I)] + \
        [(n, _D) for n in ("resorh resorm resoru resorv resorw tpeak alen depth width ratio "
                           "heatinlaser ahtoploss accul heatout heatvol beamposx beamposy "
                           "scanvel").split()] + \
        [(n, _I) for n in ("istat iend jstat jend kstat jstart powerindicator momentum_cells "
                           "fallback").split()] + [("resorc", _D), ("nk_active", _I), ("trackindx", _I), ("steadylength", _I)]

    def as_dict(self) -> Dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class AmcfdOptions(C.Structure):
    _fields_ = [("device", _I), ("order", _I), ("precision", _I), ("use_graphs", _I),
                ("check_finite", _I), ("no_small_box", _I), ("host_loop", _I),
                ("wait_polls", _I), ("autotune", _I), ("asm_kseg", _I), ("sweep_warps", _I),
                ("mom_cluster", _I), ("serial_launch", _I), ("box_ctas", _I),
                ("pass_launch", _I)]


class AmcfdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Load libamcfd_b200.so (built in-tree by __graft_entry__.build())."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python __graft_entry__.py build`")
        L = C.CDLL(LIB_PATH)
        P, VP = C.POINTER, C.c_void_p
        L.amcfd_deck_load.argtypes = [C.c_char_p, P(VP)]
        L.amcfd_deck_params.argtypes = [VP, P(AmcfdParams)]
        L.amcfd_deck_error.restype = C.c_char_p
        L.amcfd_deck_free.argtypes = [VP]
        L.amcfd_deck_string.argtypes = [VP, C.c_char_p]
        L.amcfd_deck_string.restype = C.c_char_p
        L.amcfd_sizeof_params.restype = C.c_size_t
        L.amcfd_sizeof_report.restype = C.c_size_t
        if hasattr(L, "amcfd_create"):
            L.amcfd_create.argtypes = [P(AmcfdParams), P(AmcfdOptions), P(VP)]
            L.amcfd_destroy.argtypes = [VP]
            L.amcfd_last_error.argtypes = [VP]
            L.amcfd_last_error.restype = C.c_char_p
            L.amcfd_step.argtypes = [VP, P(AmcfdReport)]
            L.amcfd_get_field.argtypes = [VP, C.c_char_p, P(_D)]
            L.amcfd_get_field_async.argtypes = [VP, C.c_char_p, P(_D)]
            L.amcfd_wait_reads.argtypes = [VP]
            L.amcfd_set_field.argtypes = [VP, C.c_char_p, P(_D)]
            L.amcfd_get_grid.argtypes = [VP, C.c_char_p, P(_D)]
            L.amcfd_dims.argtypes = [VP, P(_I), P(_I), P(_I)]
            L.amcfd_run_phase.argtypes = [VP, _I, P(AmcfdReport)]
            L.amcfd_phase_name.argtypes = [_I]
            L.amcfd_phase_name.restype = C.c_char_p
            L.amcfd_last_timing.argtypes = [VP, P(_D), _I]
            L.amcfd_profile.argtypes = [VP, _I]
            L.amcfd_free_surface.argtypes = [VP, P(AmcfdFreeSurface)]
            L.amcfd_run_steps.argtypes = [VP, _I, P(AmcfdReport), P(_D)]
            L.amcfd_tuning.argtypes = [VP, P(_I), P(_I), P(_D)]
            L.amcfd_pipe_stride.argtypes = [VP, P(_I)]
            L.amcfd_kernel_launches.argtypes = [VP]
            L.amcfd_kernel_launches.restype = C.c_longlong
            L.amcfd_run_batch.argtypes = [P(VP), _I, _I, _I, P(AmcfdReport), P(_I)]
            L.amcfd_net_param_count.restype = C.c_size_t
            L.amcfd_net_create.argtypes = [_I, C.c_ulonglong, P(VP)]
            L.amcfd_net_destroy.argtypes = [VP]
            L.amcfd_net_last_error.argtypes = [VP]
            L.amcfd_net_last_error.restype = C.c_char_p
            for f in ("get_params", "get_grads"):
                getattr(L, "amcfd_net_" + f).argtypes = [VP, P(C.c_float), C.c_size_t]
            L.amcfd_net_set_params.argtypes = [VP, P(C.c_float), C.c_size_t]
            L.amcfd_net_forward.argtypes = [VP, VP, _I, _I, _I, VP]
            L.amcfd_net_backward.argtypes = [VP, VP, P(_D)]
            L.amcfd_net_adam.argtypes = [VP, C.c_float]
            L.amcfd_net_last_ms.argtypes = [VP, P(C.c_float), P(C.c_float)]
            L.amcfd_writer_create.argtypes = [VP, VP, C.c_char_p, P(VP)]
            for f in ("step", "finish"):
                getattr(L, "amcfd_writer_" + f).argtypes = [VP]
            L.amcfd_writer_last_error.argtypes = [VP]
            L.amcfd_writer_last_error.restype = C.c_char_p
            L.amcfd_writer_destroy.argtypes = [VP]
            L.amcfd_ws_attach.argtypes = [VP, VP, _I]
            L.amcfd_ws_buffers.argtypes = [VP, P(VP), P(VP)]
            L.amcfd_ws_stats.argtypes = [VP, P(C.c_longlong), P(C.c_longlong)]
        _lib = L
    return _lib


class Deck:
    """A parsed keyword deck (amcfd_deck_load)."""

    def __init__(self, path: str):
        L = lib()
        self._h = C.c_void_p()
        rc = L.amcfd_deck_load(path.encode(), C.byref(self._h))
        if rc != 0:
            raise AmcfdError(rc, L.amcfd_deck_error().decode())
        self.path = path
        self.params = AmcfdParams()
        rc = L.amcfd_deck_params(self._h, C.byref(self.params))
        if rc != 0:
            raise AmcfdError(rc, L.amcfd_deck_error().decode())

    def string(self, what: str) -> Optional[str]:
        r = lib().amcfd_deck_string(self._h, what.encode())
        return None if r is None else r.decode()

    @property
    def dims(self):
        p = self.params
        ni = int(sum(p.ncvx[q] for q in range(p.nzx))) + 2
        nj = int(sum(p.ncvy[q] for q in range(p.nzy))) + 2
        nk = int(sum(p.ncvz[q] for q in range(p.nzz))) + 2
        return ni, nj, nk

    def close(self):
        if self._h:
            lib().amcfd_deck_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Writer:
    """The reference's output files for a run (amcfd_writer_*): .vts/.pvd,
    _Residuals.txt and the final-geometry file, under `root` (default: the
    working directory)."""

    def __init__(self, solver: "Solver", deck: "Deck", root: Optional[str] = None):
        self._solver, self._deck = solver, deck
        self._h = C.c_void_p()
        rc = lib().amcfd_writer_create(solver._h, deck._h, root.encode() if root else None, C.byref(self._h))
        if rc != 0:
            raise AmcfdError(rc, lib().amcfd_writer_last_error(self._h).decode() if self._h else "writer")

    def _check(self, rc: int) -> int:
        if rc < 0:
            raise AmcfdError(rc, lib().amcfd_writer_last_error(self._h).decode())
        return rc

    def step(self) -> bool:
        """After each Solver.step(); True when an output was written."""
        return self._check(lib().amcfd_writer_step(self._h)) == 1

    def finish(self):
        self._check(lib().amcfd_writer_finish(self._h))

    def close(self):
        if self._h:
            lib().amcfd_writer_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Net:
    """The warm-start network (amcfd_net_*).  Device arrays are passed as raw
    pointers (e.g. torch.Tensor.data_ptr()) of FP32 channels-last data."""

    def __init__(self, device: int = 0, seed: int = 1):
        self._h = C.c_void_p()
        rc = lib().amcfd_net_create(device, seed, C.byref(self._h))
        if rc != 0:
            raise AmcfdError(rc, lib().amcfd_net_last_error(self._h).decode() if self._h else "create failed")
        self.nparams = int(lib().amcfd_net_param_count())

    def _check(self, rc: int):
        if rc != 0:
            raise AmcfdError(rc, lib().amcfd_net_last_error(self._h).decode())

    def params(self) -> np.ndarray:
        out = np.empty(self.nparams, dtype=np.float32)
        self._check(lib().amcfd_net_get_params(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), self.nparams))
        return out

    def set_params(self, p: np.ndarray):
        a = np.ascontiguousarray(p, dtype=np.float32)
        self._check(lib().amcfd_net_set_params(self._h, a.ctypes.data_as(C.POINTER(C.c_float)), self.nparams))

    def grads(self) -> np.ndarray:
        out = np.empty(self.nparams, dtype=np.float32)
        self._check(lib().amcfd_net_get_grads(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), self.nparams))
        return out

    def set_grads(self, g: np.ndarray):
        """Replace the gradients the next adam() applies (amcfd_net_set_grads)."""
        a = np.ascontiguousarray(g, dtype=np.float32)
        self._check(lib().amcfd_net_set_grads(self._h, a.ctypes.data_as(C.POINTER(C.c_float)), self.nparams))

    def forward(self, feat_ptr: int, dims, y_ptr: int = 0):
        ni, nj, nk = dims
        self._check(lib().amcfd_net_forward(self._h, feat_ptr, ni, nj, nk, y_ptr or None))

    def backward(self, target_ptr: int) -> float:
        loss = C.c_double()
        self._check(lib().amcfd_net_backward(self._h, target_ptr, C.byref(loss)))
        return loss.value

    def adam(self, lr: float):
        self._check(lib().amcfd_net_adam(self._h, lr))

    def last_ms(self):
        """(forward ms, backward ms) of the last passes, from CUDA events."""
        f, b = C.c_float(), C.c_float()
        self._check(lib().amcfd_net_last_ms(self._h, C.byref(f), C.byref(b)))
        return f.value, b.value

    def close(self):
        if self._h:
            lib().amcfd_net_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_batch(solvers: Sequence["Solver"], nsteps: int, nthreads: int = 0):
    """amcfd_run_batch: nsteps steps of every solver, concurrently on one GPU.
    Returns (reports, status codes) in the order of `solvers`; raises on the first
    failure after all instances have finished."""
    n = len(solvers)
    hs = (C.c_void_p * max(n, 1))(*[s._h for s in solvers])
    reps = (AmcfdReport * max(n, 1))()
    st = (_I * max(n, 1))()
    rc = lib().amcfd_run_batch(hs, n, nsteps, nthreads, reps, st)
    if rc != 0:
        q = next(i for i in range(n) if st[i] != 0)
        raise AmcfdError(rc, f"instance {q}: " + lib().amcfd_last_error(solvers[q]._h).decode())
    return [reps[q].as_dict() for q in range(n)], [st[q] for q in range(n)]


class Solver:
    """One melt-pool instance on one GPU (amcfd_create ... amcfd_destroy).

    small_box: None lets the solver choose the momentum path of a small melt-pool
    box, 1 forces the one-CTA chain whenever the box fits, 0 never takes it."""

    def __init__(self, deck: Deck, order: int = ORDER_EXACT, precision: int = PREC_FP64,
                 device: int = 0, use_graphs: int = 0, check_finite: int = 1,
                 small_box: Optional[int] = None, host_loop: int = 0, wait_polls: int = 0, autotune: int = 0,
                 asm_kseg: int = 0, sweep_warps: int = 0, mom_cluster: int = 0, serial_launch: int = 0,
                 box_ctas: int = 0, pass_launch: int = 0):
        L = lib()
        self.deck = deck  # keeps toolpath storage alive
        opts = AmcfdOptions(device=device, order=order, precision=precision,
                            use_graphs=use_graphs, check_finite=check_finite,
                            no_small_box=0 if small_box is None else (-1 if small_box else 1), host_loop=host_loop,
                            wait_polls=wait_polls, autotune=autotune, asm_kseg=asm_kseg,
                            sweep_warps=sweep_warps, mom_cluster=mom_cluster,
                            serial_launch=serial_launch, box_ctas=box_ctas, pass_launch=pass_launch)
        self._h = C.c_void_p()
        rc = L.amcfd_create(C.byref(deck.params), C.byref(opts), C.byref(self._h))
        if rc != 0:
            msg = L.amcfd_last_error(self._h).decode() if self._h else "create failed"
            raise AmcfdError(rc, msg)
        ni, nj, nk = C.c_int(), C.c_int(), C.c_int()
        L.amcfd_dims(self._h, C.byref(ni), C.byref(nj), C.byref(nk))
        self.shape = (nk.value, nj.value, ni.value)
        self.report = AmcfdReport()

    def _check(self, rc: int):
        if rc != 0:
            raise AmcfdError(rc, lib().amcfd_last_error(self._h).decode())

    def step(self) -> Dict:
        self._check(lib().amcfd_step(self._h, C.byref(self.report)))
        return self.report.as_dict()

    def run_phase(self, phase) -> Dict:
        ph = PHASES[phase] if isinstance(phase, str) else int(phase)
        self._check(lib().amcfd_run_phase(self._h, ph, C.byref(self.report)))
        return self.report.as_dict()

    def get(self, name: str) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        self._check(lib().amcfd_get_field(self._h, name.encode(),
                                          out.ctypes.data_as(C.POINTER(_D))))
        return out

    def set(self, name: str, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(self.shape)
        self._check(lib().amcfd_set_field(self._h, name.encode(), a.ctypes.data_as(C.POINTER(_D))))

    def grid(self, name: str) -> np.ndarray:
        n = {"x": 2, "xu": 2, "y": 1, "yv": 1, "z": 0, "zw": 0}[name]
        out = np.empty(self.shape[n], dtype=np.float64)
        self._check(lib().amcfd_get_grid(self._h, name.encode(), out.ctypes.data_as(C.POINTER(_D))))
        return out

    def run_steps(self, n: int):
        """n time steps; returns (last report, device milliseconds of the n steps)."""
        ms = C.c_double()
        self._check(lib().amcfd_run_steps(self._h, n, C.byref(self.report), C.byref(ms)))
        return self.report.as_dict(), ms.value

    def profile(self, enable: bool = True):
        self._check(lib().amcfd_profile(self._h, 1 if enable else 0))

    def tuning(self) -> Dict:
        """Launch shapes in use (amcfd_tuning, amcfd_pipe_stride): assembly planes per
        CTA, lines per CTA of the per-pass sweeps, the planes between passes of the
        pipelined sweep (0 when not pipelined) and, after autotuning, the
        candidates' times in ms (sweep_ms keyed by stride when pipelined)."""
        a, w = _I(), _I()
        t = (_D * 6)()
        self._check(lib().amcfd_tuning(self._h, C.byref(a), C.byref(w), t))
        d = _I()
        self._check(lib().amcfd_pipe_stride(self._h, C.byref(d)))
        keys = (8, 16, 32) if d.value else (2, 4, 8)
        return {"asm_kseg": a.value, "sweep_warps": w.value, "pipe_stride": d.value,
                "asm_ms": {4: t[0], 8: t[1], 16: t[2]}, "sweep_ms": dict(zip(keys, t[3:6]))}

    @property
    def launches(self) -> int:
        return int(lib().amcfd_kernel_launches(self._h))

    def get_into(self, name: str, ptr: int):
        """Copy a field into caller memory at address `ptr` (ni*nj*nk doubles)."""
        self._check(lib().amcfd_get_field(self._h, name.encode(), C.cast(ptr, C.POINTER(_D))))

    def get_into_async(self, name: str, ptr: int):
        """Queue the copy of a field into caller memory at `ptr` (ni*nj*nk doubles,
        pinned for overlap) and return; the memory holds the field after wait_reads()."""
        self._check(lib().amcfd_get_field_async(self._h, name.encode(), C.cast(ptr, C.POINTER(_D))))

    def wait_reads(self):
        """Block until the last get_into_async copy has landed."""
        self._check(lib().amcfd_wait_reads(self._h))

    def ws_attach(self, net: Optional["Net"], mode: int):
        """Attach the warm-start network (WS_OFF, WS_PREDICT, WS_RECORD)."""
        self._net = net
        self._check(lib().amcfd_ws_attach(self._h, net._h if net is not None else None, mode))

    def ws_buffers(self):
        """Device pointers of the last step's features [ncell][11] and scaled
        increments [ncell][2] (FP32)."""
        f, t = C.c_void_p(), C.c_void_p()
        self._check(lib().amcfd_ws_buffers(self._h, C.byref(f), C.byref(t)))
        return f.value, t.value

    def ws_stats(self):
        a, r = C.c_longlong(), C.c_longlong()
        self._check(lib().amcfd_ws_stats(self._h, C.byref(a), C.byref(r)))
        return a.value, r.value

    TIMING_SLOTS = ("energy_assemble", "factor", "energy_sweeps", "h2t_meltpool", "momentum",
                    "converge", "laser", "update", "outer_iters", "sweep_launches", "species")

    def free_surface(self) -> Dict:
        """amcfd_free_surface: the energy-balance free surface on the current state."""
        r = AmcfdFreeSurface()
        self._check(lib().amcfd_free_surface(self._h, C.byref(r)))
        return {name: getattr(r, name) for name, _ in r._fields_}

    def timing(self, n: int = 16) -> Dict:
        out = np.zeros(n, dtype=np.float64)
        lib().amcfd_last_timing(self._h, out.ctypes.data_as(C.POINTER(_D)), n)
        return {k: float(out[q]) for q, k in enumerate(self.TIMING_SLOTS)}

    def close(self):
        if self._h:
            lib().amcfd_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
