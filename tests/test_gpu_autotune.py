"""Autotuner: InitMem times candidate launch shapes on the device (pair-kernel CTAs per
SM, PME brick edge, gather kernel) and keeps the fastest.  Every shape it can
pick gives bit-identical forces, energies and trajectories, because forces, charge
grids and energies are integer sums; this checks the defaults, the tuned shapes and
forced shapes against one another: the prune as a warp per i-block and as a CTA per
i-block (the same inner lists), and the PME spread through per-brick shared-memory
regions and straight into the grid with no brick lists (the same integer grid).
"""
import os

import numpy as np
import pytest

import fenzi_b200 as fz
from tests.helpers import system

pytestmark = pytest.mark.gpu

KNOBS = ("FZ_AUTOTUNE", "FZ_NB_CTAS_PER_SM", "FZ_PME_BRICK", "FZ_PME_GATHER", "FZ_PRUNE_SPLIT")
SHAPES = [
    {"FZ_AUTOTUNE": "0"},
    {},
    {"FZ_NB_CTAS_PER_SM": "2", "FZ_PME_BRICK": "4", "FZ_PME_GATHER": "1", "FZ_PRUNE_SPLIT": "1"},
    {"FZ_NB_CTAS_PER_SM": "3", "FZ_PME_BRICK": "16", "FZ_PME_GATHER": "2", "FZ_PRUNE_SPLIT": "0"},
    {"FZ_NB_CTAS_PER_SM": "4", "FZ_PME_GATHER": "3"},
]


def run(path, env, steps=10):
    saved = {k: os.environ.get(k) for k in KNOBS}
    for k in KNOBS:
        os.environ.pop(k, None)
    os.environ.update(env)
    try:
        s = fz.FenZi.ReadInput(path).LoadSystem()
        s.InitMem(0)
        shapes = s.launch_shapes()
        s.ComputeAccelGPU(energies=True)
        f = s.forces_fixed()
        e = s.EvalProps()
        s.InitVelocity(T=300.0, seed=9)
        s.SingleStep(steps)
        pos = s.positions()
        s.close()
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return shapes, f, e, pos


@pytest.mark.parametrize("key", ["small", "mid"])
def test_every_shape_bit_identical(key):
    _, path = system(key)
    runs = [run(path, env) for env in SHAPES]
    assert not runs[0][0]["autotuned"]
    assert runs[1][0]["autotuned"]
    assert runs[2][0]["nb_ctas_per_sm"] == 2 and runs[2][0]["pme_brick"] == [4, 4, 4]
    assert runs[3][0]["nb_ctas_per_sm"] == 3 and runs[3][0]["gather"] == "atom"
    assert runs[4][0]["gather"] == "atom-spread"
    shapes0, f0, e0, p0 = runs[0]
    assert np.any(f0 != 0)
    for shapes, f, e, p in runs[1:]:
        assert np.array_equal(f, f0), shapes
        assert e["potential"] == e0["potential"], shapes
        assert np.array_equal(p, p0), shapes
