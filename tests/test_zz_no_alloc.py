"""fz_pme_reciprocal_static: PME for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc (code inside another framework's memory pool or a
pre-sized arena).  The no-allocation entry point runs the PME kernels on fixed
file-scope device scratch; here its output is checked against the system path
(fz_compute_forces_terms with FZ_TERM_PME) on the same positions, on two calls in a
row (the shared scratch keeps the previous call's contents, so the second call also
checks that each call starts clean).  Device buffers are owned by the test (torch),
as a real caller's would be.  Kept in a file of its own that is collected last.
"""
import numpy as np
import pytest

import fenzi_b200 as fz
from tests.helpers import rel_rms, system

pytestmark = pytest.mark.gpu


def test_pme_static_matches_system_path():
    import torch
    _, path = system("small")
    s = fz.FenZi.ReadInput(path).LoadSystem()
    s.InitMem(0)
    s.ComputeAccelGPU(terms=fz.TERM_PME, energies=True)
    n = s.n
    ref = s.forces_fixed().astype(np.float64).reshape(3, n).T / 2.0 ** 32
    e_ref = s.EvalProps()["pme"]
    pos = s.positions()
    q = s.topology()["q"]
    x = np.concatenate([pos, q[:, None]], axis=1).astype(np.float32)
    dev_pos = torch.from_numpy(x).cuda()
    dev_f = torch.zeros(3 * n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    box = list(s.cfg.box)
    K = list(s.cfg.pme_grid)
    for _ in range(2):
        e = fz.pme_reciprocal_static(0, dev_pos.data_ptr(), n, box, K, s.cfg.kappa, dev_f.data_ptr())
        torch.cuda.synchronize()
        f = dev_f.cpu().numpy().astype(np.float64).reshape(3, n).T / 2.0 ** 32
        assert rel_rms(f, ref) <= 5e-5
        assert abs(e - e_ref) <= max(2e-5 * abs(e_ref), 1e-3)
    s.close()


def test_pme_static_rejects_oversized_input():
    with pytest.raises(fz.FenZiError) as err:
        fz.pme_reciprocal_static(0, 0, 10, [20.0] * 3, [128, 128, 128], 0.34, 0)
    assert err.value.code == 6
