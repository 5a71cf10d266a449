"""Minimiser (the reference's MinimizeStep loop: conjugate gradient, then steepest
descent, undoing moves that raise the energy): the potential energy of a seeded
lattice start falls, constraints stay satisfied, the reported energy is the oracle's
energy of the final positions, and dynamics continues from the minimised state."""
import numpy as np
import pytest

import fenzi_b200 as fz
from oracle import oracle as O
from tests.helpers import oracle_for, system

pytestmark = pytest.mark.gpu


def test_minimize_lowers_energy_and_keeps_constraints():
    _, path = system("small")
    s = fz.FenZi.ReadInput(path).LoadSystem()
    s.InitMem(0)
    e0 = s.EvalProps()["potential"]
    k, e = s.Minimize(300)
    assert 0 < k <= 300
    assert e < e0 - 1.0, (e0, e)
    assert abs(s.EvalProps()["potential"] - e) <= 1e-6 * abs(e) + 1e-6
    pos = s.positions()
    _, eo = oracle_for(s).forces(pos, O.T_ALL)
    assert abs(sum(eo.values()) - e) <= 2e-5 * abs(e), (sum(eo.values()), e)
    top = s.topology()
    c, d = top["cons"], top["cons_d"]
    r = pos[c[:, 0]] - pos[c[:, 1]]
    r -= np.round(r / s.cfg.box[0]) * s.cfg.box[0]
    assert np.abs(np.linalg.norm(r, axis=1) - d).max() < 1e-4
    s.InitVelocity(T=300.0, seed=8, counter=0)
    s.SingleStep(50)
    assert np.isfinite(s.EvalProps()["potential"])
    s.close()
