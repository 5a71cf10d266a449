"""The oracle pinned to the reference's own arithmetic (host only).

tests/golden/ref_terms.npz holds forces and energies computed by the reference's own
kernels (bondedforce, nonbondforce, InitDeviceConstants + BCMultiply), compiled for the
host from the reference sources by oracle/refbuild.py and run by
tests/golden/make_ref_golden.py on a seeded system that exercises every parameter
path.  Here the FP64 oracle is checked against them term by term:
  - where the reference's formulas are the oracle's (bonds, angles, Urey-Bradley,
    impropers, 1-4 pairs, the nonbonded pair without switching, dihedral energies, the
    PME influence function) they agree to rounding (1e-12);
  - where the reference departs from -dE/dr, the difference is shown to be exactly the
    departure, restated here in closed form:
      * dihedral force: the reference applies -n sin(n phi - delta) d(cos phi)/dr,
        without the factor K / sin(phi) of the energy's gradient
        (src/bonded_forces.cu:339-372);
      * LJ switch force: the reference's derivative carries an extra
        -(rc^2 - r^2)^2 Swcoeff3 Swcoeff2 / r per unit of unswitched LJ energy
        (src/nonbonded_forces.cu:204-214);
      * Ewald exclusion energy: the reference corrects a pair once per bond and once
        per angle it closes (src/bonded_forces.cu:764-768, 880-927), so the energy of a
        pair that is both (the H-H pair of a water with an H-H bond) is counted twice;
        its force once (the bond loop keeps the force only for bonds of nonzero
        force constant).
The FP32 build of the same kernels shows the reference's own single-precision error.
When oracle/_ref is built (the reference tree is present), the kernels are also run
live on a second seed.
"""
import copy
import os

import numpy as np
import pytest

import oracle.oracle as O
from oracle.oracle import Oracle
from tests.golden.make_ref_golden import GRIDS, PIN_SYSTEM, cases, evaluate, only, pin_system

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_terms.npz")
CC = 332.0716

TOL = 1e-12  # FP64 reference statements vs FP64 oracle: rounding level


@pytest.fixture(scope="module")
def pin():
    g = np.load(GOLDEN)
    _, topo, pos = pin_system()
    assert np.array_equal(g["pos"], pos), "fixture positions differ from the seeded system"
    return g, topo, pos, cases(topo)


def rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


# term -> (oracle bits, [(reference energy index, oracle energy name)])
COINCIDE = {
    "bond": (O.T_BOND, [(0, "bond")]),
    "angle": (O.T_ANGLE, [(1, "angle")]),
    "ureyb": (O.T_UREYB, [(2, "ureyb")]),
    "impr": (O.T_IMPR, [(4, "impr")]),
    "p14": (O.T_P14, [(6, "vdw"), (7, "elec")]),
    "nb_noswitch": (O.T_NB, [(0, "vdw"), (1, "elec")]),
}


@pytest.mark.parametrize("term", sorted(COINCIDE))
def test_oracle_equals_reference_where_forms_coincide(pin, term):
    g, _, pos, cs = pin
    t, _ = cs[term]
    bits, energies = COINCIDE[term]
    f, e = Oracle(t).forces(pos, bits)
    assert np.abs(f).max() > 1e-3  # the term carries force
    assert rel_rms(g[f"{term}_f64"], f) <= TOL
    for ki, name in energies:
        assert abs(g[f"{term}_e64"][ki] - e[name]) <= TOL * max(1.0, abs(e[name]))


@pytest.mark.parametrize("term", ["dihed1", "dihed2"])
def test_dihedral_energy_equals_reference(pin, term):
    g, _, pos, cs = pin
    t, _ = cs[term]
    _, e = Oracle(t).forces(pos, O.T_DIHED)
    assert abs(g[f"{term}_e64"][3] - e["dihed"]) <= TOL * abs(e["dihed"])


def _sin_phi(pos, quad, box):
    """sin(phi) with the reference's sign convention: v_k = r_{k+1} - r_k (minimum
    image), a = v1 x v2, b = v2 x v3, sin phi = (a . v3) |v2| / (|a| |b|)
    (src/bonded_forces.cu:281-297)."""
    mi = lambda d: d - np.round(d / box) * box
    v1, v2, v3 = (mi(pos[quad[k + 1]] - pos[quad[k]]) for k in range(3))
    a, b = np.cross(v1, v2), np.cross(v2, v3)
    return (a @ v3) * np.linalg.norm(v2) / (np.linalg.norm(a) * np.linalg.norm(b))


def test_dihedral_force_departure_is_k_over_sin_phi(pin):
    """Single-fold dihedrals (K 0.16, n 3, delta 0): the reference's force on every atom
    equals sum over dihedrals of (sin phi / K) x the oracle's -dE/dr of that dihedral."""
    g, topo, pos, cs = pin
    t, _ = cs["dihed1"]
    box = np.asarray(topo["box"], float)
    pred = np.zeros_like(pos)
    for d in range(len(t["dihe"])):
        td = copy.deepcopy(t)
        for key in ("dihe", "dihe_k", "dihe_n", "dihe_d"):
            td[key] = np.asarray(t[key])[d:d + 1]
        fd, _ = Oracle(td).forces(pos, O.T_DIHED)
        pred += fd * _sin_phi(pos, t["dihe"][d], box) / t["dihe_k"][d]
    assert rel_rms(g["dihed1_f64"], pred) <= TOL
    # size of the departure from -dE/dr on this system
    f, _ = Oracle(t).forces(pos, O.T_DIHED)
    assert rel_rms(g["dihed1_f64"], f) > 1.0


def test_switch_force_departure_in_closed_form(pin):
    """With the switch on (ron < r < rc) the reference's LJ force differs from -dE/dr by
    E_LJ(r) (-(rc^2 - r^2)^2 Swcoeff3 Swcoeff2 / r) d per pair; energies agree."""
    g, topo, pos, cs = pin
    t, _ = cs["nb_switch"]
    f, e = Oracle(t).forces(pos, O.T_NB)
    rc, ron = float(t["rc"]), float(t["ron"])
    sw2, sw3 = rc * rc - 3 * ron * ron, 1.0 / (rc * rc - ron * ron) ** 3
    box = np.asarray(t["box"], float)
    from oracle.ref import exclusion_pairs
    excl = exclusion_pairs(t)
    typ = np.asarray(t["type"])
    nt = int(t["ntypes"])
    eps4 = np.asarray(t["eps4"]).reshape(nt, nt)
    sig2 = np.asarray(t["sig2"]).reshape(nt, nt)
    delta = np.zeros_like(pos)
    n = len(pos)
    for i in range(n):
        d = pos[i] - pos[i + 1:]
        d -= np.round(d / box) * box
        r2 = (d * d).sum(1)
        for k in np.nonzero((r2 < rc * rc) & (r2 > ron * ron))[0]:
            j = i + 1 + int(k)
            if (i, j) in excl:
                continue
            r = np.sqrt(r2[k])
            s6 = (sig2[typ[i], typ[j]] / r2[k]) ** 3
            elj = eps4[typ[i], typ[j]] * (s6 * s6 - s6)
            a = rc * rc - r2[k]
            x = elj * (-a * a * sw3 * sw2 / r) * d[k]
            delta[i] += x
            delta[j] -= x
    assert rel_rms(g["nb_switch_f64"], f + delta) <= TOL
    assert rel_rms(g["nb_switch_f64"], f) > 1e-4  # the departure is visible
    assert abs(g["nb_switch_e64"][0] - e["vdw"]) <= TOL * abs(e["vdw"])
    assert abs(g["nb_switch_e64"][1] - e["elec"]) <= TOL * abs(e["elec"])


def test_exclusion_correction_force_equals_oracle_energy_counts_bonds_and_angles(pin):
    """The reference's Ewald exclusion correction: its force is the oracle's (each
    excluded pair once: the bond loop drops the force for bonds of zero force constant,
    src/bonded_forces.cu:767), its energy the oracle's plus one more correction for every
    pair that is both a bond and an angle's 1-3 pair (here the 100 water H-H pairs,
    whose H-H bond has K = 0)."""
    g, topo, pos, cs = pin
    t, _ = cs["ewexcl"]
    f, e = Oracle(t).forces(pos, O.T_EXCL)
    assert rel_rms(g["ewexcl_f64"], f) <= TOL
    bonds = {tuple(sorted(b)) for b in np.asarray(t["bond"]).tolist()}
    both = sorted({tuple(sorted((a, c))) for a, _, c in np.asarray(t["angle"]).tolist()} & bonds)
    assert len(both) == PIN_SYSTEM["nw"]
    t2 = only(t, ("bond",))
    t2.update(bond=np.asarray(both, np.int32), bond_k=np.zeros(len(both)), bond_r0=np.ones(len(both)))
    _, e2 = Oracle(t2).forces(pos, O.T_EXCL)
    assert abs(g["ewexcl_e64"][5] - (e["ewexcl"] + e2["ewexcl"])) <= TOL * abs(e["ewexcl"])


@pytest.mark.parametrize("grid", GRIDS, ids=lambda x: "x".join(map(str, x[0])))
def test_pme_influence_function_equals_reference(grid):
    """BCMultiply's factor x pi K^3 (the reference's cuFFT normalisation) is the oracle's
    C(m) = |b(m)|^2 exp(-pi^2 m^2 / beta^2) / m^2 on every grid point."""
    g = np.load(GOLDEN)
    K, L = grid
    tag = "x".join(str(k) for k in K)
    go = O.pme_influence(K, L, 0.34)
    gr = g[f"influence_{tag}_64"] * np.pi * np.prod(K)
    assert np.abs(gr - go).max() <= TOL * np.abs(go).max()
    g32 = g[f"influence_{tag}_32"].astype(np.float64) * np.pi * np.prod(K)
    assert np.abs(g32 - go).max() <= 1e-6 * np.abs(go).max()


def test_reference_fp32_is_within_the_real_space_bar(pin):
    """The reference's own FP32 arithmetic vs its FP64 statements: the scale of the
    1e-5 relative-RMS bar the product is held to."""
    g = pin[0]
    for term in list(COINCIDE) + ["dihed1", "dihed2", "ewexcl", "nb_switch"]:
        assert rel_rms(g[f"{term}_f32"], g[f"{term}_f64"]) <= 1e-5, term


_REF_BUILT = os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                                         "libfzref64.so"))


@pytest.mark.skipif(not _REF_BUILT, reason="oracle/_ref not built (needs the reference tree)")
def test_live_reference_kernels_second_seed():
    """The same relations with the reference kernels run live on other displacements."""
    from oracle import ref as R
    _, topo, pos0 = pin_system()
    pos = pos0 + np.random.default_rng(99).normal(0.0, 0.03, pos0.shape)
    cs = cases(topo)
    for term in ("bond", "angle", "ureyb", "impr", "p14", "nb_noswitch"):
        t, kind = cs[term]
        fr, _ = evaluate(t, pos, kind, 64)
        f, _ = Oracle(t).forces(pos, COINCIDE[term][0])
        assert rel_rms(fr, f) <= TOL, term
    K, L = (5, 6, 9), (11.0, 13.0, 17.0)
    assert np.abs(R.pme_influence(K, L, 0.3) * np.pi * np.prod(K) - O.pme_influence(K, L, 0.3)).max() <= \
        TOL * np.abs(O.pme_influence(K, L, 0.3)).max()
