"""Pins the FP64 oracle (no GPU): the reference ships no golden energies or forces,
so the oracle is checked against identities -- forces are minus the gradient of its
energies, PME converges to a direct Ewald sum, its FFT equals numpy's, SHAKE/RATTLE
satisfy their constraints, FP64 velocity Verlet conserves energy."""
import numpy as np
import pytest

from fenzi_b200 import gen_system
from oracle import oracle as O


@pytest.fixture(scope="module")
def cov():
    s = gen_system.build(name="custom", nw=80, nchains=2, chain_len=12, box=16.0, kgrid=16, rc=7.0, ron=5.5,
                         seed=21, extras=True)
    return s, O.Oracle(gen_system.topology(s))


@pytest.mark.parametrize("shape", [(16, 16, 16), (18, 20, 25), (27, 12, 10), (48, 5, 7)])
def test_fft_matches_numpy(shape):
    rng = np.random.default_rng(0)
    a = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    np.testing.assert_allclose(O.fft3d(a, -1), np.fft.fftn(a), atol=1e-9 * np.abs(a).sum())
    np.testing.assert_allclose(O.fft3d(a, +1), np.fft.ifftn(a) * a.size, atol=1e-9 * np.abs(a).sum())


TERMS = [("nb", O.T_NB), ("excl", O.T_EXCL), ("p14", O.T_P14), ("bond", O.T_BOND), ("angle", O.T_ANGLE),
         ("ureyb", O.T_UREYB), ("dihed", O.T_DIHED), ("impr", O.T_IMPR), ("pme", O.T_PME)]


@pytest.mark.parametrize("name,terms", TERMS)
def test_forces_are_minus_energy_gradient(cov, name, terms):
    s, orc = cov
    f, _ = orc.forces(s.pos, terms)
    rng = np.random.default_rng(3)
    # atoms that carry this term (chains for bonded terms)
    cand = np.arange(24) if name in ("p14", "ureyb", "dihed", "impr", "bond", "angle") else rng.choice(s.n, 8, False)
    h = 1e-5
    for i in cand[:8]:
        for c in range(3):
            p1, p2 = s.pos.copy(), s.pos.copy()
            p1[i, c] += h
            p2[i, c] -= h
            fd = -(sum(orc.forces(p1, terms)[1].values()) - sum(orc.forces(p2, terms)[1].values())) / (2 * h)
            assert abs(fd - f[i, c]) <= 2e-5 * max(1.0, abs(f[i, c])), (name, i, c, fd, f[i, c])


def test_pme_converges_to_direct_ewald():
    s = gen_system.build(name="custom", nw=300, box=None, kgrid=20, rc=8.0, ron=6.5, seed=7)
    topo = gen_system.topology(s)
    ref_f, ref_e = O.Oracle(topo).ewald_recip(s.pos, 40)
    errs = []
    for K in (20, 32, 48):
        topo["K"] = np.array([K, K, K])
        f, e = O.Oracle(topo).forces(s.pos, O.T_PME)
        errs.append(np.sqrt(((f - ref_f) ** 2).sum() / (ref_f ** 2).sum()))
        assert abs(e["pme"] - ref_e) < 0.01 * abs(ref_e)
    assert errs[0] > errs[1] > errs[2] and errs[2] < 3e-4, errs


def test_shake_and_rattle_satisfy_constraints(cov):
    s, orc = cov
    topo = orc.topo
    rng = np.random.default_rng(5)
    v = rng.normal(scale=0.3, size=s.pos.shape)
    p1 = s.pos + 0.02 * rng.normal(size=s.pos.shape)
    p, v2, bad = orc.shake(s.pos, p1, v, 0.001, tol=1e-20, maxit=100)
    assert bad == 0
    c, d = topo["cons"], topo["cons_d"]
    r = p[c[:, 0]] - p[c[:, 1]]
    r -= np.round(r / s.box) * s.box
    assert np.abs(np.linalg.norm(r, axis=1) - d).max() < 1e-10
    v3 = orc.rattle(p, v2)
    dv = v3[c[:, 0]] - v3[c[:, 1]]
    assert np.abs((dv * r).sum(1)).max() < 1e-10


def test_counter_based_normals():
    z = O.normals(50000, 1234, 7)
    assert abs(z.mean()) < 0.02 and abs(z.std() - 1) < 0.02
    assert not np.array_equal(z, O.normals(50000, 1234, 8))
    assert np.array_equal(z, O.normals(50000, 1234, 7))


def test_oracle_velocity_verlet_conserves_energy(cov):
    s, orc = cov
    v = orc.reassign_velocities(s.pos, 300.0, 11, 0)
    run = orc.md(s.pos, v, 200, dt_ps=0.0005, tol=1e-12)
    tot = run["epot"] + run["ekin"]
    assert run["bad"] == 0
    assert np.ptp(tot[50:]) < 0.02 * run["ekin"].mean(), (np.ptp(tot), run["ekin"].mean())


def test_pair_count_matches_brute_force():
    s = gen_system.build(name="custom", nw=100, box=16.0, kgrid=16, rc=6.0, ron=5.0, seed=4)
    orc = O.Oracle(gen_system.topology(s))
    d = s.pos[:, None, :] - s.pos[None, :, :]
    d -= np.round(d / s.box) * s.box
    r2 = (d ** 2).sum(-1)
    iu = np.triu_indices(s.n, 1)
    mol = np.arange(s.n) // 3
    close = (r2[iu] < 36.0) & (mol[iu[0]] != mol[iu[1]])
    assert orc.count_pairs(s.pos, 6.0) == int(close.sum())


@pytest.fixture(scope="module")
def npt_sys():
    # beta 0.6: erfc(beta rc) ~ 3e-9, so the real-space cutoff step does not spoil the
    # finite-difference virial
    s = gen_system.build(name="custom", nw=80, nchains=1, chain_len=12, box=16.0, kgrid=16, rc=7.0, ron=5.5,
                         beta=0.6, seed=23)
    return s, gen_system.topology(s)


def test_virial_fd_matches_bond_sum(npt_sys):
    """-L_a dU/dL_a of the bond energy equals sum f_a d_a over the bonds."""
    s, topo = npt_sys
    orc = O.Oracle(topo)
    w = orc.virial_fd(s.pos, 1e-6, O.T_BOND)
    b = topo["bond"]
    d = s.pos[b[:, 0]] - s.pos[b[:, 1]]
    d -= np.round(d / topo["box"]) * topo["box"]
    r = np.linalg.norm(d, axis=1)
    f = -2.0 * topo["bond_k"] * (r - topo["bond_r0"]) / r
    ref = (f[:, None] * d * d).sum(0)
    np.testing.assert_allclose(w, ref, rtol=1e-6, atol=1e-6)


def _enthalpy(topo, run, pos, vel, pref_atm, pmass):
    t = dict(topo)
    t["box"] = np.asarray(run["box"], float)
    o = O.Oracle(t)
    _, e = o.forces(pos)
    L, Ldot = run["box"][0], run["lstate"][0]
    V = float(np.prod(run["box"]))
    rho = (run["box"][1] / L) * (run["box"][2] / L)
    return sum(e.values()) + o.kinetic(vel) + pref_atm * 1.4586e-5 * V + 0.5 * pmass * rho * (3 * L * L * Ldot) ** 2


def test_oracle_npt_conserves_enthalpy(npt_sys):
    """Andersen barostat (oracle): H = U + KE + Pref V + piston KE stays flat while the
    box moves (by ~5% here: the lattice start is far from 1 atm)."""
    s, topo = npt_sys
    orc = O.Oracle(topo)
    v = orc.reassign_velocities(s.pos, 300.0, 5, 0)
    P0 = orc.group_pressure(s.pos, v)  # atm
    pmass = 2e-5
    L0 = topo["box"][0]
    lacc = (P0 - 1.0) * 1.4586e-5 / (3 * pmass * L0 * L0)
    state = dict(pos=s.pos.copy(), vel=v, box=np.array(topo["box"], float), lstate=np.array([0.0, lacc]))
    hs, Ls = [], []
    for _ in range(8):
        run = orc.npt(state["pos"], state["vel"], state["box"], state["lstate"], 15, dt_ps=0.0005, tol=1e-12,
                      pref_atm=1.0, pmass=pmass)
        assert run["bad"] == 0
        state = run
        hs.append(_enthalpy(topo, run, run["pos"], run["vel"], 1.0, pmass))
        Ls.append(run["box"][0])
    ke = orc.kinetic(state["vel"])
    assert np.ptp(hs) < 3e-3 * ke, (np.ptp(hs), ke)
    assert np.ptp(Ls) > 0.1, Ls  # the box moved


def test_atomic_and_group_pressure_agree_for_rigid_water():
    """For rigid units (SHAKE-constrained TIP3P) the atomic pressure, with the
    instantaneous constraint virial, equals the pressure of the unit centres at every
    instant: the intra-unit virial is exactly -2 x the internal kinetic energy."""
    s = gen_system.build(name="custom", nw=90, nchains=0, box=14.5, kgrid=16, rc=6.5, ron=5.0, beta=0.65, seed=29)
    orc = O.Oracle(gen_system.topology(s))
    v = orc.reassign_velocities(s.pos, 300.0, 9, 0)
    pa, _ = orc.pressure(s.pos, v)
    pg = orc.group_pressure(s.pos, v)
    assert abs(pa - pg) < 1e-3 * max(abs(pg), 100.0), (pa, pg)
