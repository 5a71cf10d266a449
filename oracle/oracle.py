"""ctypes wrapper of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU
baseline / reference leg of bench.py.  The product (fenzi_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

E_NAMES = ["bond", "angle", "ureyb", "dihed", "impr", "vdw", "elec", "pme", "ewexcl", "ewself"]
T_NB, T_EXCL, T_P14, T_PME = 1, 2, 4, 8
T_BOND, T_ANGLE, T_UREYB, T_DIHED, T_IMPR, T_SELF = 16, 32, 64, 128, 256, 512
T_ALL = 1023
T_REAL = T_NB  # nonbonded real space only


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def _lib():
    if not os.path.exists(_LIB):
        build()
    lib = C.CDLL(_LIB)
    dp = C.POINTER(C.c_double)
    lib.orc_create.restype = C.c_void_p
    lib.orc_create.argtypes = [C.c_void_p]
    lib.orc_destroy.argtypes = [C.c_void_p]
    lib.orc_forces.argtypes = [C.c_void_p, dp, dp, dp, C.c_int]
    lib.orc_ewald_recip.argtypes = [C.c_void_p, dp, C.c_int, dp, dp]
    lib.orc_fft3d.argtypes = [C.c_int, C.c_int, C.c_int, dp, C.c_int]
    lib.orc_pme_influence.argtypes = [C.POINTER(C.c_int), dp, C.c_double, dp]
    lib.orc_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    lib.orc_count_pairs.restype = C.c_longlong
    lib.orc_count_pairs.argtypes = [C.c_void_p, dp, C.c_double]
    lib.orc_shake.argtypes = [C.c_void_p, dp, dp, dp, C.c_double, C.c_double, C.c_int]
    lib.orc_rattle.argtypes = [C.c_void_p, dp, dp]
    lib.orc_kinetic.restype = C.c_double
    lib.orc_kinetic.argtypes = [C.c_void_p, dp]
    lib.orc_md.argtypes = [C.c_void_p, dp, dp, C.c_int, C.c_double, C.c_double, dp, dp, dp]
    lib.orc_minimize.argtypes = [C.c_void_p, dp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, dp,
                                 C.POINTER(C.c_int)]
    lib.orc_reassign_velocities.argtypes = [C.c_void_p, dp, C.c_double, C.c_uint64, C.c_uint32, dp]
    lib.orc_normals.argtypes = [C.c_int, C.c_uint64, C.c_uint32, dp]
    lib.orc_virial_fd.argtypes = [C.c_void_p, dp, C.c_double, C.c_int, C.c_int, dp]
    lib.orc_group_pressure.restype = C.c_double
    lib.orc_group_pressure.argtypes = [C.c_void_p, dp, dp, C.c_double]
    lib.orc_constraint_virial.argtypes = [C.c_void_p, dp, dp, dp, dp]
    lib.orc_npt.argtypes = [C.c_void_p, dp, dp, dp, dp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                            C.c_double, dp, dp]
    return lib


_lib_cache = None


def lib():
    global _lib_cache
    if _lib_cache is None:
        _lib_cache = _lib()
    return _lib_cache


class _Sys(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("q", C.c_void_p), ("mass", C.c_void_p), ("type", C.c_void_p), ("ntypes", C.c_int),
        ("eps4", C.c_void_p), ("sig2", C.c_void_p), ("eps4_14", C.c_void_p), ("sig2_14", C.c_void_p),
        ("nbond", C.c_int), ("bond", C.c_void_p), ("bond_k", C.c_void_p), ("bond_r0", C.c_void_p),
        ("nangle", C.c_int), ("angle", C.c_void_p), ("angle_k", C.c_void_p), ("angle_t0", C.c_void_p),
        ("nub", C.c_int), ("ub", C.c_void_p), ("ub_k", C.c_void_p), ("ub_r0", C.c_void_p),
        ("ndihe", C.c_int), ("dihe", C.c_void_p), ("dihe_k", C.c_void_p), ("dihe_n", C.c_void_p),
        ("dihe_d", C.c_void_p),
        ("nimpr", C.c_int), ("impr", C.c_void_p), ("impr_k", C.c_void_p), ("impr_p0", C.c_void_p),
        ("ncons", C.c_int), ("cons", C.c_void_p), ("cons_d", C.c_void_p),
        ("box", C.c_double * 3), ("rc", C.c_double), ("ron", C.c_double), ("beta", C.c_double),
        ("K", C.c_int * 3), ("nthreads", C.c_int),
    ]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """FP64 reference evaluation of one system described by a topology dict."""

    def __init__(self, topo: dict, nthreads: int = 0):
        keep = {}

        def arr(name, dtype):
            a = np.ascontiguousarray(np.asarray(topo[name]), dtype=dtype)
            keep[name] = a
            return a.ctypes.data_as(C.c_void_p)

        s = _Sys()
        s.n = int(topo["n"])
        s.q, s.mass, s.type = arr("q", np.float64), arr("mass", np.float64), arr("type", np.int32)
        s.ntypes = int(topo["ntypes"])
        s.eps4, s.sig2 = arr("eps4", np.float64), arr("sig2", np.float64)
        s.eps4_14, s.sig2_14 = arr("eps4_14", np.float64), arr("sig2_14", np.float64)
        s.nbond = len(topo["bond"])
        s.bond, s.bond_k, s.bond_r0 = arr("bond", np.int32), arr("bond_k", np.float64), arr("bond_r0", np.float64)
        s.nangle = len(topo["angle"])
        s.angle, s.angle_k, s.angle_t0 = arr("angle", np.int32), arr("angle_k", np.float64), arr("angle_t0", np.float64)
        s.nub = len(topo["ub"])
        s.ub, s.ub_k, s.ub_r0 = arr("ub", np.int32), arr("ub_k", np.float64), arr("ub_r0", np.float64)
        s.ndihe = len(topo["dihe"])
        s.dihe, s.dihe_k = arr("dihe", np.int32), arr("dihe_k", np.float64)
        s.dihe_n, s.dihe_d = arr("dihe_n", np.int32), arr("dihe_d", np.float64)
        s.nimpr = len(topo["impr"])
        s.impr, s.impr_k, s.impr_p0 = arr("impr", np.int32), arr("impr_k", np.float64), arr("impr_p0", np.float64)
        s.ncons = len(topo["cons"])
        s.cons, s.cons_d = arr("cons", np.int32), arr("cons_d", np.float64)
        for k in range(3):
            s.box[k] = float(topo["box"][k])
            s.K[k] = int(topo["K"][k])
        s.rc, s.ron, s.beta = float(topo["rc"]), float(topo["ron"]), float(topo["beta"])
        s.nthreads = nthreads
        self._keep = keep
        self._s = s
        self.n = s.n
        self.topo = topo
        self.h = lib().orc_create(C.byref(s))
        if not self.h:
            raise ValueError("oracle: constraint cluster exceeds 4 atoms / 3 constraints")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def forces(self, pos, terms=T_ALL):
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
        f = np.zeros_like(pos)
        e = np.zeros(10)
        lib().orc_forces(self.h, _dp(pos), _dp(f), _dp(e), int(terms))
        return f, dict(zip(E_NAMES, e))

    def ewald_recip(self, pos, kmax):
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
        f = np.zeros_like(pos)
        e = np.zeros(1)
        lib().orc_ewald_recip(self.h, _dp(pos), int(kmax), _dp(f), _dp(e))
        return f, float(e[0])

    def counts(self):
        out = (C.c_int * 4)()
        lib().orc_counts(self.h, out)
        return dict(ew_pairs=out[0], p14_pairs=out[1], clusters=out[2], constraints=out[3])

    def count_pairs(self, pos, rcut):
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
        return int(lib().orc_count_pairs(self.h, _dp(pos), float(rcut)))

    def shake(self, pos_ref, pos, vel, dt_ps, tol=1e-10, maxit=1000):
        pr = np.ascontiguousarray(pos_ref, np.float64)
        p = np.ascontiguousarray(pos, np.float64).copy()
        v = np.ascontiguousarray(vel, np.float64).copy()
        bad = lib().orc_shake(self.h, _dp(pr), _dp(p), _dp(v), float(dt_ps), float(tol), int(maxit))
        return p, v, bad

    def rattle(self, pos, vel):
        p = np.ascontiguousarray(pos, np.float64)
        v = np.ascontiguousarray(vel, np.float64).copy()
        lib().orc_rattle(self.h, _dp(p), _dp(v))
        return v

    def kinetic(self, vel):
        v = np.ascontiguousarray(vel, np.float64)
        return float(lib().orc_kinetic(self.h, _dp(v)))

    def md(self, pos, vel, nsteps, dt_ps=0.001, tol=1e-10, traces=True):
        p = np.ascontiguousarray(pos, np.float64).copy()
        v = np.ascontiguousarray(vel, np.float64).copy()
        f = np.zeros_like(p)
        ep = np.zeros(max(1, nsteps))
        ek = np.zeros(max(1, nsteps))
        bad = lib().orc_md(self.h, _dp(p), _dp(v), int(nsteps), float(dt_ps), float(tol), _dp(f),
                           _dp(ep) if traces else None, _dp(ek) if traces else None)
        return dict(pos=p, vel=v, f=f, epot=ep[:nsteps], ekin=ek[:nsteps], bad=bad)

    def minimize(self, pos, max_steps, cgfac=1e-10, sdfac=1e-4, cgrate=0.1, sdrate=0.01):
        """The reference's minimiser (CG then SD, moves that raise the energy undone);
        returns final positions, per-step energies and methods of the counted steps."""
        p = np.ascontiguousarray(pos, np.float64).copy()
        e = np.zeros(max(1, max_steps))
        m = np.zeros(max(1, max_steps), np.int32)
        k = lib().orc_minimize(self.h, _dp(p), int(max_steps), float(cgfac), float(sdfac), float(cgrate),
                               float(sdrate), _dp(e), m.ctypes.data_as(C.POINTER(C.c_int)))
        return dict(pos=p, steps=k, energy=e[:k], method=m[:k])

    def virial_fd(self, pos, hrel=1e-6, terms=T_ALL, group=False):
        """Diagonal virial -L_a dU/dL_a by central differences: atomic scaling, or the
        integration units' mass centres scaled with rigid units (group=True)."""
        p = np.ascontiguousarray(pos, np.float64)
        out = np.zeros(3)
        lib().orc_virial_fd(self.h, _dp(p), float(hrel), int(terms), 1 if group else 0, _dp(out))
        return out

    def group_pressure(self, pos, vel, hrel=1e-6):
        p = np.ascontiguousarray(pos, np.float64)
        v = np.ascontiguousarray(vel, np.float64)
        return float(lib().orc_group_pressure(self.h, _dp(p), _dp(v), float(hrel)))

    def constraint_virial(self, pos, vel, f):
        p = np.ascontiguousarray(pos, np.float64)
        v = np.ascontiguousarray(vel, np.float64)
        ff = np.ascontiguousarray(f, np.float64)
        out = np.zeros(3)
        lib().orc_constraint_virial(self.h, _dp(p), _dp(v), _dp(ff), _dp(out))
        return out

    def pressure(self, pos, vel, hrel=1e-6):
        """Instantaneous pressure (atm) and virial: (2 KE + W_forces + W_constraints) / (3 V)."""
        f, _ = self.forces(pos)
        w = self.virial_fd(pos, hrel) + self.constraint_virial(pos, vel, f)
        box = np.asarray(self.topo["box"], np.float64)
        V = float(np.prod(box))
        return (2.0 * self.kinetic(vel) + w.sum()) / (3.0 * V) * 68558.64100846418, w

    def npt(self, pos, vel, box, lstate, nsteps, dt_ps=0.001, tol=1e-10, pref_atm=1.0, pmass=1e-5, hrel=1e-6):
        """Andersen barostat steps; returns the final state and per-step L and P traces."""
        p = np.ascontiguousarray(pos, np.float64).copy()
        v = np.ascontiguousarray(vel, np.float64).copy()
        b = np.ascontiguousarray(box, np.float64).copy()
        ls = np.ascontiguousarray(lstate, np.float64).copy()
        Lt = np.zeros(max(1, nsteps))
        Pt = np.zeros(max(1, nsteps))
        bad = lib().orc_npt(self.h, _dp(p), _dp(v), _dp(b), _dp(ls), int(nsteps), float(dt_ps), float(tol),
                            float(pref_atm), float(pmass), float(hrel), _dp(Lt), _dp(Pt))
        return dict(pos=p, vel=v, box=b, lstate=ls, L=Lt[:nsteps], P=Pt[:nsteps], bad=bad)

    def reassign_velocities(self, pos, T, seed, counter=0):
        p = np.ascontiguousarray(pos, np.float64)
        v = np.zeros_like(p)
        lib().orc_reassign_velocities(self.h, _dp(p), float(T), int(seed), int(counter), _dp(v))
        return v


def fft3d(data, sign):
    """In-place-style 3-D complex DFT of a (nz, ny, nx) array; returns a new array."""
    a = np.ascontiguousarray(data, np.complex128).copy()
    nz, ny, nx = a.shape
    lib().orc_fft3d(nx, ny, nz, a.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)), int(sign))
    return a


def pme_influence(K, box, beta):
    """The oracle's PME influence function C(m) as a (Kz, Ky, Kx) array."""
    Ka = (C.c_int * 3)(*[int(k) for k in K])
    L = np.ascontiguousarray(box, np.float64)
    G = np.zeros(int(K[0]) * int(K[1]) * int(K[2]))
    lib().orc_pme_influence(Ka, _dp(L), float(beta), _dp(G))
    return G.reshape(int(K[2]), int(K[1]), int(K[0]))


def normals(n, seed, counter=0):
    out = np.zeros((n, 3))
    lib().orc_normals(int(n), int(seed), int(counter), _dp(out))
    return out
