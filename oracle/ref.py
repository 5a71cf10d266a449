"""ctypes front end of the reference's own force kernels compiled for the host
(oracle/_ref/libfzref{32,64}.so, built by oracle/refbuild.py from the reference
sources).  TEST INFRASTRUCTURE ONLY: it checks the oracle; the product never loads it.

`RefSystem(topo)` takes the oracle's topology dict (fenzi_b200.gen_system.topology
layout) and hands the reference kernels the same system in the reference's own
parameter conventions (restated in oracle/ref_harness.cpp).  `bonded(...)` and
`nonbond(...)` return per-atom forces and the reference's energy sums.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
BONDED_E = ["bond", "angle", "ureyb", "dihed", "impr", "ewexcl", "vdw14", "elec14"]


class _Sys(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("pos", C.c_void_p), ("q", C.c_void_p), ("type", C.c_void_p), ("ntypes", C.c_int),
        ("nbfix_eps4", C.c_void_p), ("nbfix_sig2", C.c_void_p), ("p14_eps", C.c_void_p), ("p14_sig", C.c_void_p),
        ("nbond", C.c_int), ("bond", C.c_void_p), ("bond_k", C.c_void_p), ("bond_r0", C.c_void_p),
        ("nangle", C.c_int), ("angle", C.c_void_p), ("angle_k", C.c_void_p), ("angle_t0", C.c_void_p),
        ("angle_ub", C.c_void_p), ("nub", C.c_int), ("ub_k", C.c_void_p), ("ub_s0", C.c_void_p),
        ("ndihe", C.c_int), ("dihe", C.c_void_p), ("dihe_nfold", C.c_void_p), ("fold_k", C.c_void_p),
        ("fold_n", C.c_void_p), ("fold_d", C.c_void_p),
        ("nimpr", C.c_int), ("impr", C.c_void_p), ("impr_k", C.c_void_p), ("impr_p0", C.c_void_p),
        ("box", C.c_double * 3), ("rc", C.c_double), ("ron", C.c_double), ("beta", C.c_double),
        ("nb_off", C.c_void_p), ("nb_idx", C.c_void_p),
    ]


def available(variant: int = 64) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libfzref{variant}.so"))


_libs = {}


def lib(variant: int = 64):
    if variant not in _libs:
        L = C.CDLL(os.path.join(REF_DIR, f"libfzref{variant}.so"))
        dp = C.POINTER(C.c_double)
        L.fzr_bonded.argtypes = [C.POINTER(_Sys), C.c_int, dp, dp]
        L.fzr_nonbond.argtypes = [C.POINTER(_Sys), dp, dp]
        L.fzr_pme_influence.argtypes = [C.POINTER(C.c_int), dp, C.c_double, dp]
        _libs[variant] = L
    return _libs[variant]


def pme_influence(K, box, kappa, variant=64):
    """The reference's BCMultiply factor per grid point (InitDeviceConstants moduli and
    Gaussian, divided by |m|^2 pi K^3), as a (Kz, Ky, Kx) array."""
    Ka = (C.c_int * 3)(*[int(k) for k in K])
    L = np.ascontiguousarray(box, np.float64)
    G = np.zeros(int(K[0]) * int(K[1]) * int(K[2]))
    r = lib(variant).fzr_pme_influence(Ka, L.ctypes.data_as(C.POINTER(C.c_double)), float(kappa),
                                       G.ctypes.data_as(C.POINTER(C.c_double)))
    if r != 0:
        raise RuntimeError("fzr_pme_influence: grid too large")
    return G.reshape(int(K[2]), int(K[1]), int(K[0]))


def min_image(d, box):
    return d - np.round(d / box) * box


def exclusion_pairs(topo) -> set:
    """1-2, 1-3 and 1-4 pairs (NBXMOD 5): none of them is in the nonbonded list."""
    ex = set()
    for a, b in np.asarray(topo["bond"]).reshape(-1, 2):
        ex.add((min(a, b), max(a, b)))
    for a, _, c in np.asarray(topo["angle"]).reshape(-1, 3):
        ex.add((min(a, c), max(a, c)))
    for a, _, _, d in np.asarray(topo["dihe"]).reshape(-1, 4):
        ex.add((min(a, d), max(a, d)))
    return ex


def neighbour_csr(pos, box, rlist, excl):
    """Full (both directions) list of every non-excluded pair within rlist."""
    n = len(pos)
    offs = [0]
    idx = []
    for i in range(n):
        d = min_image(pos - pos[i], box)
        r2 = (d * d).sum(1)
        js = np.nonzero(r2 < rlist * rlist)[0]
        js = [int(j) for j in js if j != i and (min(i, j), max(i, j)) not in excl]
        idx += js
        offs.append(len(idx))
    return np.asarray(offs, np.int32), np.asarray(idx, np.int32)


class RefSystem:
    """One system in the reference's conventions; arrays kept alive here."""

    def __init__(self, topo: dict, pos, rlist=None):
        self.topo = topo
        keep = {}

        def arr(name, a, dtype):
            a = np.ascontiguousarray(np.asarray(a), dtype=dtype)
            keep[name] = a
            return a.ctypes.data_as(C.c_void_p)

        n = int(topo["n"])
        self.n = n
        box = np.asarray(topo["box"], float)
        pos = np.asarray(pos, float).reshape(n, 3)
        s = _Sys()
        s.n = n
        s.pos = arr("pos", pos, np.float64)
        s.q = arr("q", topo["q"], np.float64)
        s.type = arr("type", topo["type"], np.int32)
        nt = int(topo["ntypes"])
        s.ntypes = nt
        s.nbfix_eps4 = arr("eps4", topo["eps4"], np.float64)
        s.nbfix_sig2 = arr("sig2", topo["sig2"], np.float64)
        # per-type 1-4 parameters: the 1-4 tables follow the combining rule
        # eps4 = 4 sqrt(e_i e_j), sigma^2 = (s_i + s_j)^2 (src/bonded_forces.cu:1176-1181)
        e14 = np.asarray(topo["eps4_14"], float).reshape(nt, nt)
        s14 = np.asarray(topo["sig2_14"], float).reshape(nt, nt)
        pe = np.diag(e14) / 4.0
        ps = np.sqrt(np.diag(s14)) / 2.0
        assert np.allclose(4.0 * np.sqrt(np.outer(pe, pe)), e14) and np.allclose((ps[:, None] + ps) ** 2, s14)
        s.p14_eps = arr("p14_eps", pe, np.float64)
        s.p14_sig = arr("p14_sig", ps, np.float64)
        bond = np.asarray(topo["bond"]).reshape(-1, 2)
        s.nbond = len(bond)
        s.bond, s.bond_k, s.bond_r0 = arr("bond", bond, np.int32), arr("bk", topo["bond_k"], np.float64), arr(
            "br", topo["bond_r0"], np.float64)
        ang = np.asarray(topo["angle"]).reshape(-1, 3)
        s.nangle = len(ang)
        s.angle, s.angle_k, s.angle_t0 = arr("angle", ang, np.int32), arr("ak", topo["angle_k"], np.float64), arr(
            "at", topo["angle_t0"], np.float64)
        ub = np.asarray(topo["ub"]).reshape(-1, 2)
        ubmap = {(min(a, b), max(a, b)): k for k, (a, b) in enumerate(ub)}
        aub = np.array([ubmap.get((min(a, c), max(a, c)), -1) for a, _, c in ang], np.int32)
        assert (aub >= 0).sum() == len(ub), "every Urey-Bradley pair must be the 1-3 pair of an angle"
        s.angle_ub = arr("aub", aub, np.int32)
        s.nub = len(ub)
        s.ub_k, s.ub_s0 = arr("uk", topo["ub_k"], np.float64), arr("us", topo["ub_r0"], np.float64)
        # dihedral folds: consecutive rows of the same four atoms are one dihedral
        dh = np.asarray(topo["dihe"]).reshape(-1, 4)
        quads, nfold = [], []
        for k in range(len(dh)):
            if k > 0 and np.array_equal(dh[k], dh[k - 1]):
                nfold[-1] += 1
            else:
                quads.append(dh[k])
                nfold.append(1)
        s.ndihe = len(quads)
        s.dihe = arr("dihe", np.asarray(quads).reshape(-1, 4), np.int32)
        s.dihe_nfold = arr("nfold", nfold, np.int32)
        s.fold_k, s.fold_n, s.fold_d = arr("fk", topo["dihe_k"], np.float64), arr(
            "fn", topo["dihe_n"], np.int32), arr("fd", topo["dihe_d"], np.float64)
        im = np.asarray(topo["impr"]).reshape(-1, 4)
        s.nimpr = len(im)
        s.impr, s.impr_k, s.impr_p0 = arr("impr", im, np.int32), arr("ik", topo["impr_k"], np.float64), arr(
            "ip", topo["impr_p0"], np.float64)
        for k in range(3):
            s.box[k] = float(box[k])
        s.rc, s.ron, s.beta = float(topo["rc"]), float(topo["ron"]), float(topo["beta"])
        off, idx = neighbour_csr(pos, box, float(rlist or topo["rc"]), exclusion_pairs(topo))
        s.nb_off, s.nb_idx = arr("off", off, np.int32), arr("idx", idx, np.int32)
        self.npairs = len(idx) // 2
        self._s, self._keep = s, keep

    def bonded(self, variant=64, c36=False):
        f = np.zeros((self.n, 3))
        e = np.zeros(8)
        r = lib(variant).fzr_bonded(C.byref(self._s), int(c36), f.ctypes.data_as(C.POINTER(C.c_double)),
                                    e.ctypes.data_as(C.POINTER(C.c_double)))
        if r != 0:
            raise RuntimeError(f"fzr_bonded failed ({r})")
        return f, dict(zip(BONDED_E, e))

    def nonbond(self, variant=64):
        f = np.zeros((self.n, 3))
        e = np.zeros(2)
        r = lib(variant).fzr_nonbond(C.byref(self._s), f.ctypes.data_as(C.POINTER(C.c_double)),
                                     e.ctypes.data_as(C.POINTER(C.c_double)))
        if r != 0:
            raise RuntimeError(f"fzr_nonbond failed ({r})")
        return f, dict(vdw=e[0], elec=e[1])
