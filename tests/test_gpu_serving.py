"""Serving loop: jobs admitted by an HBM budget and advanced together give the same
trajectories as the same jobs run alone (bit-identical: same kernels, int64 fixed-point
forces), NVE and NVT (velocity reassignment) jobs alike."""
import os
import tempfile

import numpy as np
import pytest

import fenzi_b200 as fz
from fenzi_b200 import gen_system

pytestmark = pytest.mark.gpu

# (waters, chains, steps, NVT)
JOBS = [(500, 0, 300, False), (800, 2, 200, True), (600, 1, 400, False), (1000, 0, 150, True),
        (700, 3, 250, False), (900, 0, 350, True)]


@pytest.fixture(scope="module")
def job_paths():
    root = tempfile.mkdtemp(prefix="fzserve_test_")
    out = []
    for i, (nw, nch, _, _) in enumerate(JOBS):
        g = gen_system.build(name=f"job{i}", nw=nw, nchains=nch, chain_len=30, rc=9.0, ron=7.5, seed=700 + i)
        out.append(gen_system.write(g, os.path.join(root, f"j{i}")))
    return out


def _load(path, nvt):
    s = fz.FenZi.ReadInput(path)
    if nvt:
        s.cfg.temp_reset_every = 100
    return s.LoadSystem()


def test_served_jobs_match_alone(job_paths):
    alone = []
    for (nw, nch, steps, nvt), path in zip(JOBS, job_paths):
        s = _load(path, nvt)
        s.InitMem(0)
        s.InitVelocity(counter=0)  # the input's temperature and seed, as the server does
        s.SingleStep(steps)
        alone.append((s.positions(), s.EvalProps()))
        s.close()
    systems = [_load(p, j[3]) for j, p in zip(JOBS, job_paths)]
    # a budget that holds about three of these jobs at once: admission must wait
    est = max(fz.Server.estimate_bytes(s) for s in systems)
    server = fz.Server(0, hbm_budget_bytes=3.2 * est, chunk_steps=64, max_running=8)
    ids = [server.submit(s, j[2]) for s, j in zip(systems, JOBS)]
    infos = [server.wait(k) for k in ids]
    stats = server.stats()
    for k, info, (pos0, e0) in zip(ids, infos, alone):
        assert info["state"] == "done" and info["steps_done"] == info["nsteps"]
        assert info["submit_s"] <= info["start_s"] <= info["end_s"]
        pos = server.positions(k)
        assert np.array_equal(pos, pos0), np.abs(pos - pos0).max()
        assert info["final"]["potential"] == e0["potential"]
        assert info["final"]["kinetic"] == e0["kinetic"]
    assert 2 <= stats["peak_running"] <= 3, stats
    assert stats["finished"] == len(JOBS)
    assert stats["atom_steps"] == sum(s * n for s, n in zip([j[2] for j in JOBS], [i["natom"] for i in infos]))
    server.close()


def test_server_rejects_job_above_budget(job_paths):
    server = fz.Server(0, hbm_budget_bytes=1e6, chunk_steps=10, max_running=2)
    k = server.submit(_load(job_paths[0], False), 10)
    with pytest.raises(fz.FenZiError) as ei:
        server.wait(k)
    assert ei.value.code == 4  # FZ_ERR_CAPACITY
    assert server.info(k)["state"] == "failed"
    server.close()
