"""Batched ensemble: every system gives the same result alone and in the batch."""
import os
import tempfile

import numpy as np
import pytest

import fenzi_b200 as fz
from fenzi_b200 import gen_system

pytestmark = pytest.mark.gpu


def _load(s, d):
    p = gen_system.write(s, d)
    sy = fz.FenZi.ReadInput(p).LoadSystem()
    sy.InitMem(0)
    sy.InitVelocity(T=300.0, seed=77)
    return sy


def test_batch_matches_each_system_alone():
    systems = gen_system.ensemble(nsys=5, seed=11, nw_min=216, nw_max=700)
    tmp = tempfile.mkdtemp(prefix="fzbatch_")
    alone = [_load(s, os.path.join(tmp, f"a{i}")) for i, s in enumerate(systems)]
    mixed = [_load(s, os.path.join(tmp, f"b{i}")) for i, s in enumerate(systems)]
    for s in alone:
        s.SingleStep(25)
    b = fz.Batch(mixed)
    b.step(25)
    for a, m in zip(alone, mixed):
        assert np.array_equal(a.positions(), m.positions())
        assert np.array_equal(a.velocities(), m.velocities())
        assert np.array_equal(a.forces_fixed(), m.forces_fixed())
    b.close()
    for s in alone + mixed:
        s.close()
