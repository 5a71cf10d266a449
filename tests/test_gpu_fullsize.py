"""Parity at the full size of the 230,400-atom workload that bench.py times (72,000 TIP3P
+ 480 x 30-atom chains, 130 A cubic box, 128^3 PME, beta 0.34, rc 10 / switch from 8).

The system first takes 200 MD steps on the device (two 100-step legs with 300 K velocity
reassignment), so the pair lists have been rebuilt and pruned there; every check then
runs at the device's own positions.

Against the FP64 oracle (relative RMS over all 230,400 atoms):
  real-space pair forces                         <= 1e-5
  bonded + 1-4 + Ewald exclusion corrections     <= 1e-5
  PME vs the FP64 PME oracle on the same mesh    <= 5e-5
Size-independent properties of the whole system:
  forces bit-identical across two evaluations (int64 fixed point);
  Newton's third law: real-space plus bonded forces sum to zero within 1e-4 of their
  root-sum-square (a single lost pair force of 1 kcal/mol/A is ~7e-5 of it);
  SHAKE/SETTLE constraints held to 5e-5 A (FP32 positions up to 65 A from the origin).
"""
import numpy as np
import pytest

import fenzi_b200 as fz
from oracle import oracle as O
from tests.helpers import ORACLE_BONDED, oracle_for, rel_rms, system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def large():
    _, path = system("large230k")
    s = fz.FenZi.ReadInput(path).LoadSystem()
    assert s.n == 230400
    s.InitMem(0)
    s.InitVelocity(T=300.0, seed=2345, counter=0)
    s.SingleStep(100)
    s.InitVelocity(T=300.0, seed=2345, counter=1)
    s.SingleStep(100)
    assert s.counters()["rebuilds"] >= 1
    yield s, oracle_for(s), s.positions()
    s.close()


@pytest.mark.parametrize("terms,oterms,tol", [
    (fz.TERM_NONBONDED, O.T_NB, 1e-5),
    (fz.TERM_BONDED, ORACLE_BONDED, 1e-5),
    (fz.TERM_PME, O.T_PME, 5e-5),
], ids=["nonbonded", "bonded", "pme"])
def test_forces_match_oracle_at_full_size(large, terms, oterms, tol):
    s, orc, pos = large
    s.ComputeAccelGPU(terms=terms)
    f = s.forces()
    f0, _ = orc.forces(pos, oterms)
    err = rel_rms(f, f0)
    print(f"full-size force error vs oracle: {err:.3e} (tolerance {tol:.0e})")
    assert err <= tol, err


def test_forces_bit_identical_and_newton3_at_full_size(large):
    s, _, _ = large
    s.ComputeAccelGPU()
    a = s.forces_fixed()
    s.ComputeAccelGPU()
    b = s.forces_fixed()
    assert np.array_equal(a, b)
    s.ComputeAccelGPU(terms=fz.TERM_NONBONDED | fz.TERM_BONDED)
    f = s.forces()
    rss = float(np.sqrt((f ** 2).sum()))
    assert rss > 0
    net = float(np.linalg.norm(f.sum(axis=0)))
    print(f"net real-space + bonded force {net:.3e}, root-sum-square {rss:.3e}")
    assert net <= 1e-4 * rss


def test_constraints_held_at_full_size(large):
    s, _, pos = large
    top = s.topology()
    c, d = top["cons"], top["cons_d"]
    r = pos[c[:, 0]] - pos[c[:, 1]]
    r -= np.round(r / s.cfg.box[0]) * s.cfg.box[0]
    dev = float(np.abs(np.linalg.norm(r, axis=1) - d).max())
    print(f"largest constraint deviation {dev:.3e} A")
    assert dev < 5e-5
