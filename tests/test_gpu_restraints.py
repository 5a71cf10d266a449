"""consharm restraint and consfix fixed segments (src/mdcuda.cu:481-516,
src/cell_based_kernels.cu:715-877, src/prmread.cu:674-723): every atom of the second
restraint segment gets fc (dist + R0 - R1) with R the segments' mass centres (positions
wrapped into the primary box), and atoms of fixed segments never move."""
import numpy as np
import pytest

import fenzi_b200 as fz
from tests.helpers import system

pytestmark = pytest.mark.gpu


def test_consharm_force_on_second_segment():
    _, path = system("small")
    base = fz.FenZi.ReadInput(path).LoadSystem()
    base.InitMem(0)
    base.ComputeAccelGPU()
    f0 = base.forces()
    pos = base.positions()
    top = base.topology()
    _, path = system("small")
    s = fz.FenZi.ReadInput(path)
    s.cfg.consharm = 1
    s.cfg.consharm_seg[0].value = b"wat"   # names compare case-insensitively
    s.cfg.consharm_seg[1].value = b"CHN"
    for d, v in enumerate((1.0, -2.0, 0.5)):
        s.cfg.consharm_dist[d] = v
    s.cfg.consharm_fc = 2.5
    s.LoadSystem()
    s.InitMem(0)
    s.set_positions(pos)
    s.ComputeAccelGPU()
    df = s.forces() - f0
    L = np.array(s.cfg.box[:3])
    w = pos - L * np.floor(pos / L + 0.5)
    m = top["mass"]
    chn = np.arange(s.n) < 20  # the generator writes the chains first (2 x 10 atoms)
    r0 = (m[~chn, None] * w[~chn]).sum(0) / m[~chn].sum()
    r1 = (m[chn, None] * w[chn]).sum(0) / m[chn].sum()
    want = 2.5 * (np.array([1.0, -2.0, 0.5]) + r0 - r1)
    assert np.abs(df[chn] - want).max() < 1e-4 * max(1.0, np.abs(want).max())
    assert np.abs(df[~chn]).max() < 1e-6
    s.close()
    base.close()


def test_consfix_segment_does_not_move():
    _, path = system("small")
    s = fz.FenZi.ReadInput(path)
    s.cfg.consfix_nseg = 1
    s.cfg.consfix_seg[0].value = b"CHN"
    s.LoadSystem()
    s.InitMem(0)
    p0 = s.positions()
    s.InitVelocity(T=300.0, seed=2, counter=0)
    assert np.abs(s.velocities()[:20]).max() == 0.0
    s.SingleStep(50)
    d = s.positions()[:20] - p0[:20]
    L = s.cfg.box[0]
    d -= np.round(d / L) * L
    assert np.abs(d).max() < 1e-5
    assert np.abs(s.positions()[20:] - p0[20:]).max() > 1e-3  # the rest moves
    s.close()
