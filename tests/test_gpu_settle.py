"""Rigid waters: SETTLE (the closed-form SHAKE solution, default for symmetric 3-atom
triangles) against the Newton SHAKE solver on the same system and start.

Both solve the same equations, so 20 steps agree to the FP32 storage of positions
(<= 1e-5 A) and every constraint holds to 1e-5 A.
"""
import os

import numpy as np
import pytest

import fenzi_b200 as fz
from tests.helpers import system

pytestmark = pytest.mark.gpu


def run(path, settle, steps=20):
    old = os.environ.get("FZ_SETTLE")
    os.environ["FZ_SETTLE"] = "1" if settle else "0"
    try:
        s = fz.FenZi.ReadInput(path).LoadSystem()
        s.InitMem(0)
    finally:
        if old is None:
            os.environ.pop("FZ_SETTLE", None)
        else:
            os.environ["FZ_SETTLE"] = old
    s.InitVelocity(T=300.0, seed=31)
    s.SingleStep(steps)
    out = s.positions(), s.velocities(), s.topology()
    s.close()
    return out


def test_settle_matches_newton_shake():
    _, path = system("small")
    p1, v1, t = run(path, True)
    p0, v0, _ = run(path, False)
    L = np.array(t["box"])
    d = p1 - p0
    d -= np.round(d / L) * L
    assert np.abs(d).max() < 1e-5, np.abs(d).max()
    assert np.abs(v1 - v0).max() < 1e-4
    c, dd = t["cons"], t["cons_d"]
    r = p1[c[:, 0]] - p1[c[:, 1]]
    r -= np.round(r / L) * L
    assert np.abs(np.linalg.norm(r, axis=1) - dd).max() < 1e-5
