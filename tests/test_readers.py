"""Drop-in readers (host only): .in keywords, CRD/PDB/XYZ, RTF+PSF, PRM, exclusions."""
import json
import os

import numpy as np
import pytest

import fenzi_b200 as fz
from fenzi_b200 import gen_system
from tests.helpers import system

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "dmpc_small.json")
# the reference's example deck: under $FENZI_REFERENCE, or the copy oracle/refbuild.py
# keeps in oracle/_ref (built from the reference tree, not committed)
_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DMPC = next((p for p in (os.path.join(os.environ.get("FENZI_REFERENCE", "-"), "tests", "examples_fenzi", "dmpc_small",
                                      "fenzi.in"),
                         os.path.join(_ROOT, "oracle", "_ref", "dmpc_small", "fenzi.in")) if os.path.exists(p)),
            "")


@pytest.mark.skipif(not DMPC, reason="reference example deck not present")
def test_dmpc_small_matches_reference_headers():
    """The reference's own complete deck: counts equal the PSF headers and an
    independent restatement of the exclusion/constraint rules (golden fixture)."""
    g = json.load(open(GOLDEN))
    s = fz.FenZi.ReadInput(DMPC)
    c = s.cfg
    assert list(c.box) == g["box"] and list(c.pme_grid) == g["pme_grid"]
    assert (c.kappa, c.cutoff, c.cuton, c.pairlistdist) == (g["kappa"], g["cutoff"], g["cuton"], g["pairlistdist"])
    assert c.shake == 1 and c.shake_tol == g["shake_tol"] and c.seed == g["seed"]
    assert c.temp_reset_every == g["temp_reset_every"] and c.unknown_keywords == 0
    s.LoadSystem()
    i = s.info()
    for k in ("natom", "nbond", "nangle", "ndihedral", "nimproper", "nexcl_pairs", "n14_pairs", "nconstraint",
              "ncluster"):
        assert getattr(i, k) == g[k], k
    t = s.topology()
    assert abs(t["q"].sum() - g["net_charge"]) < 1e-6
    assert abs(t["mass"].sum() - g["total_mass"]) < 1e-3
    # NBFIX (HT-HT, HT-OT) overrides the combining rule in the normal table only
    assert np.all(t["eps4"] >= 0) and np.all(t["sig2"] >= 0)
    assert np.allclose(t["eps4"], t["eps4"].T) and np.allclose(t["sig2"], t["sig2"].T)


def test_synthetic_round_trip():
    s, path = system("small")
    sy = fz.FenZi.ReadInput(path).LoadSystem()
    t = sy.topology()
    ref = gen_system.topology(s)
    assert np.abs(t["pos"] - s.pos).max() < 1e-5  # CRD keeps 5 decimals
    np.testing.assert_allclose(t["q"], ref["q"])
    np.testing.assert_allclose(t["mass"], ref["mass"])
    assert np.array_equal(t["bond"], ref["bond"]) and np.array_equal(t["angle"], ref["angle"])
    np.testing.assert_allclose(t["bond_k"], ref["bond_k"])
    np.testing.assert_allclose(t["bond_r0"], ref["bond_r0"], rtol=1e-14)
    np.testing.assert_allclose(t["angle_k"], ref["angle_k"])
    np.testing.assert_allclose(t["angle_t0"], ref["angle_t0"], atol=1e-6)
    np.testing.assert_allclose(t["dihe_k"], ref["dihe_k"])
    assert np.array_equal(t["dihe_n"], ref["dihe_n"])
    # LJ tables agree once both type numberings are mapped to atoms
    ti, tr = t["type"], ref["type"]
    idx = np.arange(0, s.n, 37)
    e_prod = t["eps4"][ti[idx][:, None], ti[idx][None, :]]
    e_ref = ref["eps4"][tr[idx][:, None], tr[idx][None, :]]
    np.testing.assert_allclose(e_prod, e_ref, rtol=1e-14)
    s_prod = t["sig2"][ti[idx][:, None], ti[idx][None, :]]
    s_ref = ref["sig2"][tr[idx][:, None], tr[idx][None, :]]
    np.testing.assert_allclose(s_prod, s_ref, rtol=1e-14)
    i = sy.info()
    assert i.nconstraint == len(ref["cons"]) and i.ncluster == 400
    # exclusions: waters 3 pairs each, chains 1-2 + 1-3; 1-4 = chain dihedrals
    assert i.nexcl_pairs == 3 * 400 + 2 * (9 + 8) and i.n14_pairs == 2 * 7


def test_ext_crd_and_other_coordinate_formats(tmp_path):
    s = gen_system.build(name="custom", nw=50, box=12.0, kgrid=16, rc=5.0, ron=4.0, seed=1)
    path = gen_system.write(s, str(tmp_path / "a"))
    base = fz.FenZi.ReadInput(path).LoadSystem().topology()["pos"]
    # PDB and XYZ carrying the same coordinates select their readers by extension
    pdb = tmp_path / "a" / "x.pdb"
    with open(pdb, "w") as f:
        for i, p in enumerate(base):
            f.write(f"ATOM  {i + 1:5d} OH2  TIP W{1:4d}    {p[0]:8.3f}{p[1]:8.3f}{p[2]:8.3f}  1.00  0.00\n")
    xyz = tmp_path / "a" / "x.xyz"
    with open(xyz, "w") as f:
        f.write(f"{len(base)}\ncomment\n" + "".join(f"O {p[0]:.5f} {p[1]:.5f} {p[2]:.5f}\n" for p in base))
    for cpath, tol in ((pdb, 6e-4), (xyz, 1e-5)):
        txt = open(path).read().replace("coordinates custom.crd", f"coordinates {cpath.name}")
        inp = tmp_path / "a" / f"{cpath.suffix[1:]}.in"
        inp.write_text(txt)
        p2 = fz.FenZi.ReadInput(str(inp)).LoadSystem().topology()["pos"]
        assert np.abs(p2 - base).max() < tol


def test_input_keywords_and_errors(tmp_path):
    s, path = system("small")
    txt = open(path).read()
    p = tmp_path / "k.in"
    p.write_text(txt.replace("shake on", "SHAKE on") + "tempresetTiming 20\nINBFRQ 5\nbogus 1\n"
                 "checkpointformat ascii\npmass 500\npref 2.0\n")
    c = fz.FenZi.ReadInput(str(p)).cfg
    assert c.shake == 1 and c.temp_reset_every == 20 and c.inbfrq == 5 and c.unknown_keywords == 1
    assert c.checkpointformat == b"a" and c.pmass == 500 and c.pref == 2.0
    with pytest.raises(fz.FenZiError) as e:
        fz.FenZi.ReadInput(str(tmp_path / "missing.in"))
    assert e.value.code == 1
    bad = tmp_path / "bad.in"
    bad.write_text(txt.replace(os.path.basename(path.replace("fenzi.in", "custom.prm")), "nothere.prm"))
    with pytest.raises(fz.FenZiError) as e:
        fz.FenZi.ReadInput(str(bad)).LoadSystem()
    assert e.value.code == 1


def test_missing_parameter_is_an_error(tmp_path):
    s = gen_system.build(name="custom", nw=20, nchains=1, chain_len=6, box=12.0, kgrid=16, rc=5.0, ron=4.0, seed=2)
    path = gen_system.write(s, str(tmp_path / "m"))
    prm = os.path.join(os.path.dirname(path), "custom.prm")
    txt = open(prm).read()
    open(prm, "w").write("\n".join(l for l in txt.splitlines() if not l.startswith("CTU  CTU  CTU  CTU")) + "\n")
    with pytest.raises(fz.FenZiError) as e:
        fz.FenZi.ReadInput(path).LoadSystem()
    assert e.value.code == 2 and "dihedral" in str(e.value)
