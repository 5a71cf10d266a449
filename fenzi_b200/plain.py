"""ctypes binding of the plain comparator path (include/fenzi_plain.h).

The plain path restates the reference's GPU method stage for stage (per-atom full
neighbour list, thread-per-atom nonbonded, gather-style PME spread, complex cuFFT,
one launch per stage, a host synchronisation every step) so that fenzi_b200's step
can be timed against it on the same GPU; with fp64=True every quantity is FP64 (the
all-FP64 variant of energy-drift comparisons).  Method names follow FenZi's.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import Energies, FenZi, FenZiError, _check, _dp, lib

PLAIN_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libfenzi_plain.so")
PLAIN_EXPORTS = ["fz_plain_create", "fz_plain_free", "fz_plain_set_positions", "fz_plain_set_velocities",
                 "fz_plain_get_positions", "fz_plain_get_velocities", "fz_plain_compute_forces", "fz_plain_step",
                 "fz_plain_eval_props", "fz_plain_get_counters"]
_plib = None


def plib():
    """Loads libfenzi_plain.so (after libfenzi_b200.so, whose error channel it shares)."""
    global _plib
    if _plib is None:
        lib()
        if not os.path.exists(PLAIN_LIB_PATH):
            raise ImportError(f"{PLAIN_LIB_PATH} is missing: run `python -m fenzi_b200.build`")
        L = C.CDLL(PLAIN_LIB_PATH)
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        sig = {
            "fz_plain_create": ([vp, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
            "fz_plain_free": ([vp], C.c_int),
            "fz_plain_set_positions": ([vp, dp], C.c_int),
            "fz_plain_set_velocities": ([vp, dp], C.c_int),
            "fz_plain_get_positions": ([vp, dp], C.c_int),
            "fz_plain_get_velocities": ([vp, dp], C.c_int),
            "fz_plain_compute_forces": ([vp, dp], C.c_int),
            "fz_plain_step": ([vp, C.c_int], C.c_int),
            "fz_plain_eval_props": ([vp, C.POINTER(Energies)], C.c_int),
            "fz_plain_get_counters": ([vp, C.POINTER(C.c_longlong)], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes, f.restype = args, res
        _plib = L
    return _plib


class Plain:
    """One system on the plain path, built from a loaded FenZi system (which need not
    be uploaded).  Positions start at the system's coordinates, velocities at zero."""

    def __init__(self, system: FenZi, device: int = 0, fp64: bool = False):
        if not system.h:
            raise FenZiError(7, "Plain: load the system first (LoadSystem)")
        self.fp64 = bool(fp64)
        self.h = C.c_void_p()
        _check(plib().fz_plain_create(system.h, int(device), 1 if fp64 else 0, C.byref(self.h)))
        self.n = system.n if system.n else system.info().natom

    def set_positions(self, pos):
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        _check(plib().fz_plain_set_positions(self.h, _dp(p)))

    def set_velocities(self, vel):
        v = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1)
        _check(plib().fz_plain_set_velocities(self.h, _dp(v)))

    def positions(self):
        out = np.empty((self.n, 3))
        _check(plib().fz_plain_get_positions(self.h, _dp(out)))
        return out

    def velocities(self):
        out = np.empty((self.n, 3))
        _check(plib().fz_plain_get_velocities(self.h, _dp(out)))
        return out

    def ComputeAccelGPU(self):
        out = np.empty((self.n, 3))
        _check(plib().fz_plain_compute_forces(self.h, _dp(out)))
        return out

    def SingleStep(self, nsteps: int = 1):
        _check(plib().fz_plain_step(self.h, int(nsteps)))

    def EvalProps(self) -> dict:
        e = Energies()
        _check(plib().fz_plain_eval_props(self.h, C.byref(e)))
        return e.as_dict()

    def counters(self) -> dict:
        out = (C.c_longlong * 4)()
        _check(plib().fz_plain_get_counters(self.h, out))
        return {"rebuilds": out[0], "list_entries": out[1], "steps": out[2], "launches": out[3]}

    def close(self):
        if self.h:
            plib().fz_plain_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
