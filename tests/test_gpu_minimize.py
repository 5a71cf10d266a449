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


@pytest.mark.parametrize("nsteps", [1, 2, 5, 10, 20, 40])
def test_minimize_moves_match_oracle(nsteps):
    """The first moves of fz_minimize against the oracle's FP64 restatement of the
    reference's MinimizeStep loop (CG moves with the per-atom gamma, the undo-and-switch
    rule, SD moves) on a system without constraints, from the same positions: energy
    and positions after each number of moves."""
    g, path = system("min_free", name="custom", nw=200, nchains=2, chain_len=10, rc=7.0, ron=6.0, seed=13)
    s = fz.FenZi.ReadInput(path)
    s.cfg.shake = 0
    # factors at which the third CG move raises the energy: undone, then SD moves
    s.cfg.conjgradfac = 1e-3
    s.cfg.steepdesfac = 2e-4
    s.LoadSystem()
    s.InitMem(0)
    pos0 = s.positions()
    k, e = s.Minimize(nsteps)
    orc = oracle_for(s)
    ref = orc.minimize(pos0, nsteps, cgfac=1e-3, sdfac=2e-4, cgrate=s.cfg.conjgradrate, sdrate=s.cfg.steepdesrate)
    if nsteps >= 5:
        assert list(ref["method"][:3]) == [1, 1, 2]  # the switch is exercised
    assert k == ref["steps"], (k, ref["steps"], ref["method"])
    # the potential is a small difference of large terms: tolerance on their scale
    _, terms = orc.forces(ref["pos"])
    scale = sum(abs(v) for v in terms.values())
    assert abs(e - ref["energy"][-1]) <= 2e-6 * scale, (e, ref["energy"][-1], scale)
    d = s.positions() - ref["pos"]
    d -= np.round(d / s.cfg.box[0]) * s.cfg.box[0]
    assert np.abs(d).max() <= 2e-4, np.abs(d).max()
    s.close()
