"""The plain comparator path (libfenzi_plain.so) on the GPU.

It must compute the same physics as the product path, so it is held to the FP64
oracle like the product:
  FP64 plain forces vs oracle      rel RMS <= 1e-9 (same forms and mesh; summation order only)
  FP32 plain forces vs oracle      rel RMS <= 5e-5 (FP32 arithmetic, FP32 PME mesh)
  energies per term                FP64: 1e-8 relative (1e-6 kcal/mol absolute); FP32: 1e-4 / 1e-2
  FP64 plain MD vs oracle MD       positions within 1e-6 A after 40 steps
  product path vs plain FP32       rel RMS <= 1e-4
"""
import numpy as np
import pytest

import fenzi_b200 as fz
from fenzi_b200.plain import Plain
from oracle import oracle as O
from tests.helpers import oracle_for, rel_rms, system

pytestmark = pytest.mark.gpu

PRESETS = {
    "extras": dict(name="custom", nw=300, nchains=2, chain_len=10, rc=7.0, ron=6.0, seed=17, extras=True),
    "tiny": {},
    "small": {},
}


def loaded(key):
    _, path = system(key, **PRESETS[key])
    s = fz.FenZi.ReadInput(path).LoadSystem()
    return s, oracle_for(s)


@pytest.mark.parametrize("key", ["extras", "tiny", "small"])
@pytest.mark.parametrize("fp64", [True, False])
def test_plain_forces_and_energies_match_oracle(key, fp64):
    s, orc = loaded(key)
    p = Plain(s, 0, fp64=fp64)
    pos = p.positions()
    f = p.ComputeAccelGPU()
    e = p.EvalProps()
    f0, e0 = orc.forces(pos, O.T_ALL)
    err = rel_rms(f, f0)
    assert err <= (1e-9 if fp64 else 5e-5), err
    rtol, atol = (1e-8, 1e-6) if fp64 else (1e-4, 1e-2)
    for k in O.E_NAMES:
        assert abs(e[k] - e0[k]) <= atol + rtol * abs(e0[k]), (k, e[k], e0[k])
    p.close()


def test_plain_fp64_md_follows_oracle_md():
    s, orc = loaded("extras")
    p = Plain(s, 0, fp64=True)
    pos = p.positions()
    vel = orc.reassign_velocities(pos, 300.0, 11)
    p.set_velocities(vel)
    # both integrate constrained dynamics from the same (constrained) start
    ref = orc.md(pos, vel, 40, dt_ps=s.cfg.timestep_ps, tol=1e-14)
    p.SingleStep(40)
    dx = p.positions() - ref["pos"]
    L = np.array(s.cfg.box[:3])
    dx -= np.round(dx / L) * L
    assert np.abs(dx).max() < 1e-6, np.abs(dx).max()
    p.close()


def test_plain_nve_energy_and_constraints():
    """NVE from a hot lattice start: the conserved energy of both precisions changes by
    no more than the cutoff's own error allows (bounded loosely: the two trajectories
    part after some hundred steps), and SHAKE holds the bond lengths."""
    s, orc = loaded("small")
    vel = orc.reassign_velocities(s.topology()["pos"], 300.0, 21)
    de = {}
    for fp64 in (True, False):
        p = Plain(s, 0, fp64=fp64)
        p.set_velocities(vel)
        p.SingleStep(1)
        e0 = p.EvalProps()["conserved"]
        p.SingleStep(300)
        de[fp64] = p.EvalProps()["conserved"] - e0
        t = s.topology()
        c, d = t["cons"], t["cons_d"]
        x = p.positions()
        r = x[c[:, 0]] - x[c[:, 1]]
        L = np.array(s.cfg.box[:3])
        r -= np.round(r / L) * L
        assert np.abs(np.linalg.norm(r, axis=1) - d).max() < (1e-9 if fp64 else 2e-5)
        cnt = p.counters()
        assert cnt["steps"] == 301 and cnt["rebuilds"] >= 1 and cnt["list_entries"] > 0
        p.close()
    assert abs(de[True]) < 2.0 and abs(de[False]) < 2.0, de


def test_product_path_matches_plain_fp32():
    s, _ = loaded("extras")
    p = Plain(s, 0, fp64=False)
    fp = p.ComputeAccelGPU()
    s.InitMem(0)
    s.ComputeAccelGPU()
    err = rel_rms(s.forces(), fp)
    assert err <= 1e-4, err
    p.close()
    s.close()


def test_plain_list_holds_every_pair_twice():
    """The full list keeps each pair within the pair-list radius once per atom."""
    s, orc = loaded("small")
    p = Plain(s, 0, fp64=True)
    p.ComputeAccelGPU()
    cnt = p.counters()
    rl = max(s.cfg.pairlistdist, s.cfg.cutoff)
    pairs = orc.count_pairs(p.positions(), rl)  # non-excluded pairs within rl
    assert abs(cnt["list_entries"] - 2 * pairs) <= 4, (cnt["list_entries"], 2 * pairs)
    p.close()
