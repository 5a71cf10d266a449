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


def test_batched_kernels_match_per_system_branches():
    """The batched kernels (one launch per kernel over all members) and the graph of
    per-member branches give bit-identical trajectories, on members with chains (free-
    atom and bonded-term classes besides rigid water) and odd grid sizes (25, 27)."""
    specs = [dict(nw=300, nchains=2, chain_len=10, box=24.0, kgrid=25),
             dict(nw=420, nchains=0, box=25.5, kgrid=27),
             dict(nw=260, nchains=1, chain_len=12, box=22.0, kgrid=24),
             dict(nw=500, nchains=3, chain_len=8, box=27.0, kgrid=32)]
    tmp = tempfile.mkdtemp(prefix="fzbk_")
    runs = {}
    for mode in ("1", "0"):
        old = os.environ.get("FZ_BATCH_KERNELS")
        os.environ["FZ_BATCH_KERNELS"] = mode
        try:
            sys_ = [_load(gen_system.build(name="custom", rc=9.0, ron=7.5, seed=40 + i, **sp),
                          os.path.join(tmp, f"{mode}_{i}")) for i, sp in enumerate(specs)]
            b = fz.Batch(sys_)
            b.step(30)
            runs[mode] = [(s.positions(), s.velocities(), s.forces_fixed()) for s in sys_]
            b.close()
            for s in sys_:
                s.close()
        finally:
            if old is None:
                os.environ.pop("FZ_BATCH_KERNELS", None)
            else:
                os.environ["FZ_BATCH_KERNELS"] = old
    for (p1, v1, f1), (p0, v0, f0) in zip(runs["1"], runs["0"]):
        assert np.array_equal(p1, p0)
        assert np.array_equal(v1, v0)
        assert np.array_equal(f1, f0)
