"""Multi-step CUDA graphs: fz_step and fz_batch_step replay one graph per 100 steps
(chunks never straddle a velocity reassignment); the trajectory is bit-identical to
one graph launch per step (FZ_GRAPH_CHUNK=1), with and without NVT reassignments."""
import numpy as np
import pytest

import fenzi_b200 as fz
from fenzi_b200 import gen_system
from tests.helpers import system

pytestmark = pytest.mark.gpu


def _run(monkeypatch, chunk, nsteps, reset_every=0):
    monkeypatch.setenv("FZ_GRAPH_CHUNK", str(chunk))
    _, path = system("small")
    s = fz.FenZi.ReadInput(path)
    s.cfg.temp_reset_every = reset_every
    s.LoadSystem()
    s.InitMem(0)
    s.InitVelocity(T=300.0, seed=31, counter=0)
    s.SingleStep(nsteps)
    out = s.positions(), s.velocities(), s.counters()
    s.close()
    return out


@pytest.mark.parametrize("reset_every", [0, 150])
def test_chunked_graph_bit_identical(monkeypatch, reset_every):
    p1, v1, _ = _run(monkeypatch, 1, 430, reset_every)
    p2, v2, c2 = _run(monkeypatch, 100, 430, reset_every)
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)


def test_batch_chunked_graph_bit_identical(monkeypatch):
    systems = gen_system.ensemble(nsys=6, seed=77)
    import os
    import tempfile
    root = tempfile.mkdtemp(prefix="fz_chunk_")
    paths = [gen_system.write(g, os.path.join(root, f"b{i}")) for i, g in enumerate(systems)]
    res = []
    for chunk in (1, 100):
        monkeypatch.setenv("FZ_GRAPH_CHUNK", str(chunk))
        ss = []
        for p in paths:
            s = fz.FenZi.ReadInput(p).LoadSystem()
            s.InitMem(0)
            s.InitVelocity(T=300.0, seed=5, counter=0)
            ss.append(s)
        b = fz.Batch(ss)
        b.step(250)
        res.append([s.positions() for s in ss])
        b.close()
        for s in ss:
            s.close()
    for a, c in zip(*res):
        assert np.array_equal(a, c)
