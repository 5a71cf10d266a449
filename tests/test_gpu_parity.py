"""GPU parity: every sm_100a kernel against the FP64 oracle on the same seeded inputs.

Tolerances (relative RMS over all atoms, sqrt(sum|F-F0|^2 / sum|F0|^2)):
  real-space pair forces      <= 1e-5   (FP32 pair arithmetic, int64 accumulation)
  bonded + 1-4 + exclusions   <= 1e-5
  PME vs the FP64 PME oracle  <= 5e-5   (FP32 spline/FFT arithmetic on the same mesh)
  energies (per term)         <= 2e-5 relative (or 1e-3 kcal/mol absolute)
"""
import numpy as np
import pytest

import fenzi_b200 as fz
from oracle import oracle as O
from tests.helpers import ORACLE_BONDED, oracle_for, rel_rms, system

pytestmark = pytest.mark.gpu

_LOADED = {}


def gpu_system(key):
    if key not in _LOADED:
        _, path = system(key)
        s = fz.FenZi.ReadInput(path).LoadSystem()
        s.InitMem(0)
        _LOADED[key] = (s, oracle_for(s))
    return _LOADED[key]


@pytest.mark.parametrize("key", ["small", "water3000", "mid"])
def test_nonbonded_matches_oracle(key):
    s, orc = gpu_system(key)
    s.ComputeAccelGPU(terms=fz.TERM_NONBONDED)
    f = s.forces()
    f0, _ = orc.forces(s.positions(), O.T_NB)
    err = rel_rms(f, f0)
    assert err <= 1e-5, err


@pytest.mark.parametrize("key", ["small", "mid"])
def test_bonded_matches_oracle(key):
    s, orc = gpu_system(key)
    s.ComputeAccelGPU(terms=fz.TERM_BONDED)
    f = s.forces()
    f0, _ = orc.forces(s.positions(), ORACLE_BONDED)
    err = rel_rms(f, f0)
    assert err <= 1e-5, err


@pytest.mark.parametrize("key", ["small", "water3000"])
def test_pme_matches_oracle(key):
    s, orc = gpu_system(key)
    s.ComputeAccelGPU(terms=fz.TERM_PME)
    f = s.forces()
    f0, _ = orc.forces(s.positions(), O.T_PME)
    err = rel_rms(f, f0)
    assert err <= 5e-5, err


@pytest.mark.parametrize("K", [6, 10, 12])
def test_pme_small_and_odd_grids(K):
    """Grids of one brick per dimension (K = 6: the spread region wraps onto its own
    brick), of edge-5 bricks (K = 10) and of edge-4 bricks (K = 12); all three use
    the runtime FFT plan (no compile-time kernel for these sizes)."""
    _, path = system(f"tiny_k{K}", name="custom", nw=60, nchains=1, chain_len=8, box=14.0, kgrid=K, rc=6.0,
                     ron=5.0, seed=3)
    s = fz.FenZi.ReadInput(path).LoadSystem()
    s.InitMem(0)
    orc = oracle_for(s)
    s.ComputeAccelGPU(terms=fz.TERM_PME)
    f = s.forces()
    f0, _ = orc.forces(s.positions(), O.T_PME)
    err = rel_rms(f, f0)
    assert err <= 5e-5, err
    s.close()


def test_pme_vs_direct_ewald():
    """PME force error against a converged direct Ewald sum, relative to the total
    electrostatic force (real space + reciprocal): 3,000 TIP3P in 44.8 A, 48^3, beta 0.34."""
    s, orc = gpu_system("water3000")
    s.ComputeAccelGPU(terms=fz.TERM_PME)
    f = s.forces()
    pos = s.positions()
    fe, _ = orc.ewald_recip(pos, 30)
    fr, _ = orc.forces(pos, O.T_NB | O.T_EXCL | O.T_P14)
    err = float(np.sqrt(((f - fe) ** 2).sum() / ((fr + fe) ** 2).sum()))
    assert err <= 8e-4, err  # order-4 smooth PME at 0.93 A spacing (FP64 mesh: 5.6e-4)


def test_energies_match_oracle():
    s, orc = gpu_system("small")
    e = s.EvalProps()
    _, e0 = orc.forces(s.positions(), O.T_ALL)
    for k in ["bond", "angle", "dihed", "vdw", "elec", "pme", "ewexcl", "ewself"]:
        assert abs(e[k] - e0[k]) <= max(2e-5 * abs(e0[k]), 1e-3), (k, e[k], e0[k])


def test_total_forces_bit_reproducible():
    s, _ = gpu_system("water3000")
    s.ComputeAccelGPU()
    a = s.forces_fixed()
    s.ComputeAccelGPU()
    b = s.forces_fixed()
    assert np.array_equal(a, b)


def test_velocity_reassignment_matches_oracle():
    s, orc = gpu_system("small")
    s.InitVelocity(T=300.0, seed=2345, counter=0)
    v = s.velocities()
    v0 = orc.reassign_velocities(s.positions(), 300.0, 2345, 0)
    assert rel_rms(v, v0) <= 1e-6


def test_steps_match_oracle():
    """10 velocity-Verlet + SHAKE/RATTLE steps from the same state."""
    _, path = system("small")
    s = fz.FenZi.ReadInput(path).LoadSystem()
    s.InitMem(0)
    orc = oracle_for(s)
    s.InitVelocity(T=300.0, seed=99, counter=0)
    p0, v0 = s.positions(), s.velocities()
    s.SingleStep(10)
    p, v = s.positions(), s.velocities()
    ref = orc.md(p0, v0, 10, dt_ps=0.001, tol=1e-10)
    d = p - ref["pos"]
    d -= np.round(d / s.cfg.box[0]) * s.cfg.box[0]
    assert np.abs(d).max() < 2e-4, np.abs(d).max()
    assert rel_rms(v, ref["vel"]) < 1e-3
    # constraints hold
    top = s.topology()
    c, dd = top["cons"], top["cons_d"]
    r = p[c[:, 0]] - p[c[:, 1]]
    r -= np.round(r / s.cfg.box[0]) * s.cfg.box[0]
    assert np.abs(np.linalg.norm(r, axis=1) - dd).max() < 2e-5
    s.close()


def test_steps_bit_reproducible():
    _, path = system("water3000")
    outs = []
    for _ in range(2):
        s = fz.FenZi.ReadInput(path).LoadSystem()
        s.InitMem(0)
        s.InitVelocity(T=300.0, seed=5, counter=0)
        s.SingleStep(30)
        outs.append((s.positions(), s.forces_fixed()))
        s.close()
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def test_nve_energy_conservation():
    _, path = system("small")
    s = fz.FenZi.ReadInput(path).LoadSystem()
    s.InitMem(0)
    s.InitVelocity(T=300.0, seed=1, counter=0)
    s.SingleStep(50)  # let the lattice start relax
    e0 = s.EvalProps()
    tot0 = e0["potential"] + e0["kinetic"]
    es = []
    for _ in range(10):
        s.SingleStep(20)
        e = s.EvalProps()
        es.append(e["potential"] + e["kinetic"])
    drift = max(abs(x - tot0) for x in es)
    # fluctuation bound: a small fraction of the kinetic energy
    assert drift < 0.02 * e0["kinetic"], (drift, e0["kinetic"])
    s.close()
