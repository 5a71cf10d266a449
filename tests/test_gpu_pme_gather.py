"""PME force gather: the per-brick kernel (the brick's potential region staged in
shared memory) and the per-atom kernel (grid read from global memory) sum the same
64 terms per atom in the same order, so their int64 force buffers are bit-identical
(the launcher picks one by the mean atoms per brick; FZ_PME_GATHER forces either).
"""
import os

import numpy as np
import pytest

import fenzi_b200 as fz
from tests.helpers import system

pytestmark = pytest.mark.gpu


def run(path, mode, steps):
    old = os.environ.get("FZ_PME_GATHER")
    os.environ["FZ_PME_GATHER"] = mode
    try:
        s = fz.FenZi.ReadInput(path).LoadSystem()
        s.InitMem(0)
        s.ComputeAccelGPU(terms=fz.TERM_PME)
        f = s.forces_fixed()
        s.InitVelocity(T=300.0, seed=5)
        s.SingleStep(steps)
        pos = s.positions()
        s.close()
    finally:
        if old is None:
            os.environ.pop("FZ_PME_GATHER", None)
        else:
            os.environ["FZ_PME_GATHER"] = old
    return f, pos


@pytest.mark.parametrize("key", ["small", "mid"])
def test_brick_and_atom_gather_identical(key):
    _, path = system(key)
    fb, pb = run(path, "1", 10)
    fa, pa = run(path, "2", 10)
    assert np.any(fb != 0)
    assert np.array_equal(fb, fa)
    assert np.array_equal(pb, pa)
