"""fz_pme_reciprocal_static: PME for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc (code inside another framework's memory pool or a
pre-sized arena).  The no-allocation entry point runs the PME kernels on fixed
file-scope device scratch; here its output is checked against the FP64 oracle's PME on
the same mesh and against the system path (fz_compute_forces_terms with FZ_TERM_PME) on
the same positions, on two calls in a row (the shared scratch keeps the previous call's
contents, so the second call also checks that each call starts clean), and on a
non-cubic grid of 8 x 12 x 15 points (bricks of 4 x 4 x 5, three or fewer per axis).
Device buffers are owned by the test (torch), as a real caller's would be.  Kept in a
file of its own that is collected last.
"""
import numpy as np
import pytest

import fenzi_b200 as fz
from oracle.oracle import T_PME, Oracle
from tests.helpers import rel_rms, system

pytestmark = pytest.mark.gpu

# FP32 mesh arithmetic vs the FP64 oracle on the same mesh (the system path's PME bar)
TOL_ORACLE = 5e-5
# the system path and this entry point run the same kernels on the same FP32 tables
TOL_SELF = 1e-6


def _run_static(pos, q, box, K, beta):
    import torch
    n = len(pos)
    x = np.concatenate([pos, q[:, None]], axis=1).astype(np.float32)
    dev_pos = torch.from_numpy(x).cuda()
    dev_f = torch.zeros(3 * n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    out = []
    for _ in range(2):
        e = fz.pme_reciprocal_static(0, dev_pos.data_ptr(), n, list(box), list(K), beta, dev_f.data_ptr())
        torch.cuda.synchronize()
        out.append((dev_f.cpu().numpy().astype(np.float64).reshape(3, n).T / 2.0 ** 32, e))
    return out


def test_pme_static_matches_oracle_and_system_path():
    s_gen, path = system("small")
    s = fz.FenZi.ReadInput(path).LoadSystem()
    s.InitMem(0)
    s.ComputeAccelGPU(terms=fz.TERM_PME, energies=True)
    n = s.n
    ref = s.forces_fixed().astype(np.float64).reshape(3, n).T / 2.0 ** 32
    e_ref = s.EvalProps()["pme"]
    pos = s.positions()
    from fenzi_b200 import gen_system
    f_orc, e_orc = Oracle(gen_system.topology(s_gen)).forces(pos, T_PME)
    box, K = list(s.cfg.box), list(s.cfg.pme_grid)
    for f, e in _run_static(pos, s_gen.charge, box, K, s.cfg.kappa):
        assert rel_rms(f, f_orc) <= TOL_ORACLE
        assert abs(e - e_orc["pme"]) <= 2e-5 * abs(e_orc["pme"])
        assert rel_rms(f, ref) <= TOL_SELF
        assert abs(e - e_ref) <= 1e-6 * abs(e_ref)
    s.close()


def test_pme_static_noncubic_grid_matches_oracle():
    s_gen, _ = system("tiny")
    topo = dict(__import__("fenzi_b200").gen_system.topology(s_gen))
    box = [14.0, 15.0, 17.0]
    K = [8, 12, 15]
    topo["box"], topo["K"] = np.asarray(box), np.asarray(K, np.int32)
    pos = s_gen.pos - np.floor(s_gen.pos / np.asarray(box) + 0.5) * np.asarray(box)
    f_orc, e_orc = Oracle(topo).forces(pos, T_PME)
    for f, e in _run_static(pos, s_gen.charge, box, K, 0.34):
        assert rel_rms(f, f_orc) <= TOL_ORACLE
        assert abs(e - e_orc["pme"]) <= 2e-5 * abs(e_orc["pme"])


def test_pme_static_rejects_oversized_input():
    with pytest.raises(fz.FenZiError) as err:
        fz.pme_reciprocal_static(0, 0, 10, [20.0] * 3, [128, 128, 128], 0.34, 0)
    assert err.value.code == 6
