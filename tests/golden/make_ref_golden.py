"""Generates tests/golden/ref_terms.npz: forces and energies computed by the
reference's OWN kernels (src/bonded_forces.cu bondedforce, src/nonbonded_forces.cu
nonbondforce, src/cell_based_kernels.cu InitDeviceConstants + BCMultiply), compiled
for the host from the reference sources by oracle/refbuild.py, on a seeded system.

The system: fenzi_b200.gen_system.build(**PIN_SYSTEM) with every parameter path of the
extras preset (bonds, angles, Urey-Bradley, two-fold dihedrals with delta 0 and 30
degrees, impropers, NBFIX, special 1-4 LJ), positions displaced by seeded N(0, 0.05 A)
noise so that every bonded term carries a force.  Each term is evaluated alone
(every other term removed from the topology, charges zeroed where they would add the
Ewald exclusion correction; the 1-4 pairs and the exclusion correction, which the
reference computes inside its dihedral, bond and angle loops, as the difference of the
loops with and without charges), in the FP64 build (the reference's statements in double,
for comparison with the FP64 oracle at rounding level) and the FP32 build (the
reference's own single-precision arithmetic).

Run (needs the reference tree): python oracle/refbuild.py && python tests/golden/make_ref_golden.py
"""
import copy
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from fenzi_b200 import gen_system  # noqa: E402
from oracle import ref as R  # noqa: E402

PIN_SYSTEM = dict(name="custom", nw=100, nchains=3, chain_len=10, box=16.0, kgrid=16, rc=7.0, ron=5.5, seed=5,
                  extras=True)
NOISE = (1, 0.05)  # seed, standard deviation (A)
GRIDS = [((16, 16, 16), (16.0, 16.0, 16.0)), ((8, 12, 15), (20.0, 23.0, 27.0))]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_terms.npz")


def pin_system():
    """(gen_system.System, topology dict, displaced positions)."""
    s = gen_system.build(**PIN_SYSTEM)
    topo = gen_system.topology(s)
    rng = np.random.default_rng(NOISE[0])
    pos = s.pos + rng.normal(0.0, NOISE[1], s.pos.shape)
    return s, topo, pos


_E2, _E3, _E4, _E0 = (np.zeros((0, 2), np.int32), np.zeros((0, 3), np.int32), np.zeros((0, 4), np.int32),
                      np.zeros(0))


def only(topo, keep, charges=True, lj14=True, single_fold=False):
    """The topology with every bonded term not in `keep` removed."""
    t = copy.deepcopy(topo)
    if "bond" not in keep:
        t.update(bond=_E2, bond_k=_E0, bond_r0=_E0)
    if "angle" not in keep:
        t.update(angle=_E3, angle_k=_E0, angle_t0=_E0)
    if "ub" not in keep:
        t.update(ub=_E2, ub_k=_E0, ub_r0=_E0)
    if "dihe" not in keep:
        t.update(dihe=_E4, dihe_k=_E0, dihe_n=np.zeros(0, np.int32), dihe_d=_E0)
    if "impr" not in keep:
        t.update(impr=_E4, impr_k=_E0, impr_p0=_E0)
    if not charges:
        t["q"] = np.zeros(t["n"])
    if not lj14:
        t["eps4_14"] = np.zeros_like(t["eps4_14"])
    if single_fold:
        # the first fold of every dihedral (K 0.16, n 3, delta 0)
        k = np.asarray([i for i in range(len(t["dihe"])) if i == 0 or not np.array_equal(t["dihe"][i], t["dihe"][i - 1])])
        for key in ("dihe", "dihe_k", "dihe_n", "dihe_d"):
            t[key] = np.asarray(t[key])[k]
    return t


def cases(topo):
    """name -> (topology, kind): the terms evaluated one at a time."""
    c = {
        "bond": (only(topo, ("bond",), charges=False), "bonded"),
        "angle": (only(topo, ("angle",), charges=False), "bonded"),
        "impr": (only(topo, ("impr",), charges=False), "bonded"),
        "dihed1": (only(topo, ("dihe",), charges=False, lj14=False, single_fold=True), "bonded"),
        "dihed2": (only(topo, ("dihe",), charges=False, lj14=False), "bonded"),
        "p14": (only(topo, ("dihe",)), "bonded_minus_dihed"),
    }
    t = only(topo, ("angle", "ub"), charges=False)
    t["angle_k"] = np.zeros_like(t["angle_k"])
    c["ureyb"] = (t, "bonded")
    c["ewexcl"] = (only(topo, ("bond", "angle")), "bonded_minus_uncharged")
    t = copy.deepcopy(topo)
    t["ron"] = t["rc"]
    c["nb_noswitch"] = (t, "nonbond")
    c["nb_switch"] = (copy.deepcopy(topo), "nonbond")
    return c


def evaluate(topo, pos, kind, variant):
    if kind == "nonbond":
        f, e = R.RefSystem(topo, pos).nonbond(variant)
        return f, np.array([e["vdw"], e["elec"]])
    f, e = R.RefSystem(topo, pos).bonded(variant)
    ev = np.array([e[k] for k in R.BONDED_E])
    if kind in ("bonded_minus_dihed", "bonded_minus_uncharged"):
        # the 1-4 pairs are evaluated inside the reference's dihedral loop and the Ewald
        # exclusion correction inside its bond and angle loops (its force only for bonds
        # of nonzero force constant, src/bonded_forces.cu:767): subtract the same loops
        # without charges (and 1-4 LJ), on which the bonded forces do not depend
        t0 = copy.deepcopy(topo)
        t0["q"] = np.zeros(t0["n"])
        if kind == "bonded_minus_dihed":
            t0["eps4_14"] = np.zeros_like(t0["eps4_14"])
        f0, e0 = R.RefSystem(t0, pos).bonded(variant)
        f = f - f0
        ev = ev - np.array([e0[k] for k in R.BONDED_E])
    return f, ev


def main():
    if not (R.available(64) and R.available(32)):
        sys.exit("oracle/_ref/libfzref{32,64}.so missing: run python oracle/refbuild.py first")
    _, topo, pos = pin_system()
    out = {"pos": pos}
    for name, (t, kind) in cases(topo).items():
        for v in (64, 32):
            f, e = evaluate(t, pos, kind, v)
            out[f"{name}_f{v}"] = f
            out[f"{name}_e{v}"] = e
    for K, L in GRIDS:
        tag = "x".join(str(k) for k in K)
        out[f"influence_{tag}_64"] = R.pme_influence(K, L, PIN_SYSTEM.get("beta", 0.34), 64)
        out[f"influence_{tag}_32"] = R.pme_influence(K, L, PIN_SYSTEM.get("beta", 0.34), 32).astype(np.float32)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()
