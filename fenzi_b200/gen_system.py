"""Seeded synthetic CHARMM systems (TIP3P water boxes, optionally with linear chains).

Writes the same input set the reference reads (``.in`` run file, ``.crd``, ``.psf``,
``.prm``, ``.rtf``) so the drop-in readers are exercised, and returns the exact
topology it wrote as numpy arrays (the independent description used by the tests).

Workloads (box edges in Angstrom):
  water3000   3,000 TIP3P, 44.8 A box, 48^3 PME, rc 10 / ron 8, beta 0.34
  large230k   72,000 TIP3P + 480 x 30-atom chains = 230,400 atoms, 130 A box, 128^3
  chain17k    5,360 TIP3P + 40 chains = 17,280 atoms, 56 A box, 64^3
  ensemble    waters in 216..2000 at 0.0334 A^-3, grid = smallest 2^a3^b5^c >= L/1.2, rc 9
The reference ships only example decks (tests/examples_fenzi/*); there is no public
benchmark set, so these seeded systems stand in for the workloads named above.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

# TIP3P as in CHARMM (LJ on hydrogens), geometry O-H 0.9572, H-O-H 104.52
ROH = 0.9572
THOH = 104.52
RHH = 2.0 * ROH * math.sin(math.radians(THOH / 2.0))  # 1.5139
TYPES = {
    # name: (mass, eps, rmin/2)
    "OT": (15.9994, 0.1521, 1.7682),
    "HT": (1.008, 0.046, 0.2245),
    "CTU": (14.027, 0.078, 2.05),  # united-atom chain bead
}
RTF_IDS = {"HT": 4, "OT": 75, "CTU": 81}
CHAIN_BOND = (222.5, 1.53)
CHAIN_ANGLE = (58.35, 111.0)
CHAIN_DIHE = (0.16, 3, 0.0)
# parameter-coverage extras (exercise UB, impropers, NBFIX, multi-fold dihedrals, 1-4 LJ)
EXTRA_UB = (12.0, 2.52)
EXTRA_DIHE2 = (0.05, 1, 30.0)
EXTRA_IMPR = (1.5, 0.0)
EXTRA_NBFIX = (0.12, 3.7)          # CTU-OT emin, rmin
EXTRA_14 = (0.05, 1.9)             # CTU 1-4 eps, rmin/2
WATER_BOND = (450.0, ROH)
WATER_HH = (0.0, round(RHH, 4))  # as written to the PRM (8.4f)
WATER_ANGLE = (55.0, THOH)


@dataclass
class System:
    name: str
    box: np.ndarray                      # (3,)
    pos: np.ndarray                      # (n,3) float64
    types: list                          # per-atom type name
    charge: np.ndarray
    mass: np.ndarray
    atom_names: list
    resnames: list
    segids: list
    resids: np.ndarray
    bonds: np.ndarray                    # (nb,2) 0-based
    angles: np.ndarray                   # (na,3)
    dihedrals: np.ndarray                # (nd,4)
    impropers: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int64))
    kgrid: tuple = (48, 48, 48)
    rc: float = 10.0
    ron: float = 8.0
    beta: float = 0.34
    pairlist: float = 11.0
    temperature: float = 300.0
    timestep: float = 0.001
    seed: int = 2345
    shake_tol: float = 1e-10
    extras: bool = False

    @property
    def n(self):
        return len(self.types)


def fft_friendly(n: int) -> int:
    """Smallest 2^a 3^b 5^c >= n."""
    m = max(1, int(math.ceil(n)))
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def _random_rotations(rng, n):
    # uniform random unit quaternions (Shoemake)
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a = np.sqrt(1 - u1)
    b = np.sqrt(u1)
    q = np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2),
                  b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)], axis=1)
    w, x, y, z = q[:, 3], q[:, 0], q[:, 1], q[:, 2]
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _water_local():
    h = math.radians(THOH / 2.0)
    return np.array([[0.0, 0.0, 0.0],
                     [ROH * math.sin(h), 0.0, ROH * math.cos(h)],
                     [-ROH * math.sin(h), 0.0, ROH * math.cos(h)]])


class _Grid:
    """Hash grid for rejection tests during chain growth."""

    def __init__(self, box, cell):
        self.box = np.asarray(box, float)
        self.nc = np.maximum(1, (self.box // cell).astype(int))
        self.cell = self.box / self.nc
        self.cells = {}

    def _key(self, p):
        c = np.floor((p - np.floor(p / self.box) * self.box) / self.cell).astype(int) % self.nc
        return tuple(c)

    def add(self, p, tag):
        self.cells.setdefault(self._key(p), []).append((np.array(p), tag))

    def too_close(self, p, r, skip=()):
        k = np.array(self._key(p))
        r2 = r * r
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    key = tuple((k + (dx, dy, dz)) % self.nc)
                    for q, tag in self.cells.get(key, ()):
                        if tag in skip:
                            continue
                        d = p - q
                        d -= self.box * np.round(d / self.box)
                        if d @ d < r2:
                            return True
        return False


def _grow_chains(rng, box, nchains, nlen, clash=2.5):
    grid = _Grid(box, 3.0)
    out = np.zeros((nchains, nlen, 3))
    b, th = CHAIN_BOND[1], math.radians(CHAIN_ANGLE[1])
    for c in range(nchains):
        for attempt in range(200):
            atoms = []
            p0 = rng.random(3) * box
            if grid.too_close(p0, clash):
                continue
            atoms.append(p0)
            ok = True
            for k in range(1, nlen):
                placed = False
                for _ in range(60):
                    if k == 1:
                        v = rng.normal(size=3)
                        v /= np.linalg.norm(v)
                        p = atoms[0] + b * v
                    else:
                        a1 = atoms[k - 1] - atoms[k - 2]
                        a1 /= np.linalg.norm(a1)
                        if k == 2:
                            t = rng.normal(size=3)
                        else:
                            t = atoms[k - 3] - atoms[k - 2]
                        n1 = np.cross(a1, t)
                        n1 /= np.linalg.norm(n1)
                        n2 = np.cross(n1, a1)
                        phi = rng.random() * 2 * np.pi
                        d = (-math.cos(th)) * a1 + math.sin(th) * (math.cos(phi) * n2 + math.sin(phi) * n1)
                        p = atoms[k - 1] + b * d
                    own = {(c, j) for j in range(max(0, k - 3), k)}
                    if grid.too_close(p, clash, skip=own):
                        continue
                    # clash with own earlier atoms beyond 1-4
                    bad = False
                    for j in range(0, k - 3):
                        d = p - atoms[j]
                        if d @ d < clash * clash:
                            bad = True
                            break
                    if bad:
                        continue
                    atoms.append(p)
                    placed = True
                    break
                if not placed:
                    ok = False
                    break
            if ok:
                for j, p in enumerate(atoms):
                    grid.add(p, (c, j))
                out[c] = np.array(atoms)
                break
        else:
            raise RuntimeError("chain growth failed; box too crowded")
    return out


def _place_waters(rng, box, nw, chain_atoms, excl=2.5, jitter=0.2):
    """TIP3P oxygens on a cubic lattice (finest lattice that still leaves nw free sites
    after removing sites within `excl` of chain atoms), random subset, +-jitter."""
    L = float(box[0])
    n0 = max(1, int(math.ceil(nw ** (1.0 / 3.0))))
    ca = np.asarray(chain_atoms, float).reshape(-1, 3)
    for n in range(n0, n0 + 40):
        s = L / n
        keep = np.ones((n, n, n), bool)
        if len(ca):
            # lattice index of each chain atom, then test the +-r neighbourhood of sites
            u = (ca + L / 2) / s - 0.5
            base = np.floor(u).astype(int)
            r = int(math.ceil(excl / s)) + 1
            offs = np.arange(-r, r + 1)
            ox, oy, oz = np.meshgrid(offs, offs, offs, indexing="ij")
            off = np.stack([ox.ravel(), oy.ravel(), oz.ravel()], 1)
            for o in off:
                idx = base + o
                site = (idx + 0.5) * s - L / 2
                d = site - ca
                d -= L * np.round(d / L)
                hit = (d * d).sum(1) < excl * excl
                ii = idx[hit] % n
                keep[ii[:, 0], ii[:, 1], ii[:, 2]] = False
        g = (np.arange(n) + 0.5) * s - L / 2
        sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1)[keep]
        if len(sites) >= nw:
            sel = np.sort(rng.choice(len(sites), nw, replace=False))
            return sites[sel] + rng.uniform(-jitter, jitter, size=(nw, 3))
    raise RuntimeError("could not place waters")


def build(name="water3000", seed=2345, nw=None, nchains=0, box=None, kgrid=None, rc=10.0, ron=8.0,
          beta=0.34, chain_len=30, pairlist=None, temperature=300.0, extras=False):
    """Build one seeded system.  Named presets override the keyword sizes."""
    presets = {
        "water3000": dict(nw=3000, nchains=0, box=44.8, kgrid=48, rc=10.0, ron=8.0),
        "large230k": dict(nw=72000, nchains=480, box=130.0, kgrid=128, rc=10.0, ron=8.0),
        "chain17k": dict(nw=5360, nchains=40, box=56.0, kgrid=64, rc=10.0, ron=8.0),
    }
    if name in presets:
        p = presets[name]
        nw, nchains, box, kgrid, rc, ron = p["nw"], p["nchains"], p["box"], p["kgrid"], p["rc"], p["ron"]
    if box is None:
        box = (nw / 0.0334) ** (1.0 / 3.0)
    if kgrid is None:
        kgrid = fft_friendly(box / 1.2)
    rng = np.random.default_rng(seed)
    boxv = np.array([box, box, box], float)
    chains = _grow_chains(rng, boxv, nchains, chain_len) if nchains else np.zeros((0, chain_len, 3))
    chain_flat = chains.reshape(-1, 3)
    ow = _place_waters(rng, boxv, nw, chain_flat)
    R = _random_rotations(rng, nw)
    wl = _water_local()
    wpos = ow[:, None, :] + np.einsum("nij,kj->nki", R, wl)
    # assemble: chains first, then waters (both wrapped into [-L/2, L/2))
    pos = np.concatenate([chain_flat, wpos.reshape(-1, 3)], 0)
    pos = pos - np.floor((pos + box / 2) / box) * box
    nca = nchains * chain_len
    types = ["CTU"] * nca + ["OT", "HT", "HT"] * nw
    charge = np.concatenate([np.tile([0.09, -0.09], (nca + 1) // 2)[:nca], np.tile([-0.834, 0.417, 0.417], nw)])
    mass = np.array([TYPES[t][0] for t in types])
    atom_names = [f"C{j + 1}" for c in range(nchains) for j in range(chain_len)] + ["OH2", "H1", "H2"] * nw
    resnames = ["CHN"] * nca + ["TIP3"] * (3 * nw)
    segids = ["CHN"] * nca + ["WAT"] * (3 * nw)
    resids = np.concatenate([np.repeat(np.arange(1, nchains + 1), chain_len),
                             np.repeat(np.arange(1, nw + 1), 3)]).astype(np.int64)
    bonds, angles, dihes = [], [], []
    for c in range(nchains):
        b0 = c * chain_len
        bonds += [(b0 + j, b0 + j + 1) for j in range(chain_len - 1)]
        angles += [(b0 + j, b0 + j + 1, b0 + j + 2) for j in range(chain_len - 2)]
        dihes += [(b0 + j, b0 + j + 1, b0 + j + 2, b0 + j + 3) for j in range(chain_len - 3)]
    w0 = nca + 3 * np.arange(nw)
    wb = np.stack([np.stack([w0, w0 + 1], 1), np.stack([w0, w0 + 2], 1), np.stack([w0 + 1, w0 + 2], 1)], 1).reshape(-1, 2)
    wa = np.stack([w0 + 1, w0, w0 + 2], 1)
    bonds = np.concatenate([np.array(bonds, np.int64).reshape(-1, 2), wb], 0)
    angles = np.concatenate([np.array(angles, np.int64).reshape(-1, 3), wa], 0)
    dihes = np.array(dihes, np.int64).reshape(-1, 4)
    imprs = np.zeros((0, 4), np.int64)
    if extras:
        imprs = np.array([(c * chain_len + j, c * chain_len + j + 1, c * chain_len + j + 2, c * chain_len + j + 3)
                          for c in range(nchains) for j in range(0, chain_len - 3, 4)], np.int64).reshape(-1, 4)
    return System(impropers=imprs, extras=extras, name=name, box=boxv, pos=pos, types=types, charge=charge, mass=mass, atom_names=atom_names,
                  resnames=resnames, segids=segids, resids=resids, bonds=bonds, angles=angles, dihedrals=dihes,
                  kgrid=(kgrid, kgrid, kgrid), rc=rc, ron=ron, beta=beta,
                  pairlist=pairlist if pairlist is not None else rc + 1.0, temperature=temperature, seed=seed)


# ------------------------------------------------------------------ topology for the oracle
def topology(s: System):
    """Exact parameters of every term, resolved without the readers."""
    names = sorted(set(s.types), key=lambda t: RTF_IDS[t])
    tid = {t: i for i, t in enumerate(names)}
    nt = len(names)
    eps = np.array([TYPES[t][1] for t in names])
    rmh = np.array([TYPES[t][2] for t in names])
    sig_half = rmh / 2 ** (1.0 / 6.0)
    eps4 = 4.0 * np.sqrt(np.outer(eps, eps))
    sig2 = (sig_half[:, None] + sig_half[None, :]) ** 2
    typ = np.array([tid[t] for t in s.types], np.int32)
    btype = [(s.types[a], s.types[b]) for a, b in s.bonds]
    bk = np.array([WATER_HH[0] if bt == ("HT", "HT") else (WATER_BOND[0] if "OT" in bt else CHAIN_BOND[0]) for bt in btype])
    br = np.array([WATER_HH[1] if bt == ("HT", "HT") else (WATER_BOND[1] if "OT" in bt else CHAIN_BOND[1]) for bt in btype])
    is_w = np.array([s.types[a[1]] == "OT" for a in s.angles], bool)
    ak = np.where(is_w, WATER_ANGLE[0], CHAIN_ANGLE[0])
    at = np.radians(np.where(is_w, WATER_ANGLE[1], CHAIN_ANGLE[1]))
    nd = len(s.dihedrals)
    dihe, dk, dn, dd = s.dihedrals, np.full(nd, CHAIN_DIHE[0]), np.full(nd, CHAIN_DIHE[1]), np.full(nd, 0.0)
    ub = np.zeros((0, 2), np.int32)
    ubk, ubr = np.zeros(0), np.zeros(0)
    ik, ip = np.zeros(len(s.impropers)), np.zeros(len(s.impropers))
    eps4_14, sig2_14 = eps4.copy(), sig2.copy()
    if s.extras:
        # two folds per chain dihedral, in the order the PRM lists them
        dihe = np.repeat(s.dihedrals, 2, axis=0)
        dk = np.tile([CHAIN_DIHE[0], EXTRA_DIHE2[0]], nd)
        dn = np.tile([CHAIN_DIHE[1], EXTRA_DIHE2[1]], nd)
        dd = np.tile([math.radians(CHAIN_DIHE[2]), math.radians(EXTRA_DIHE2[2])], nd)
        ca = ~is_w
        ub = s.angles[ca][:, [0, 2]].astype(np.int32)
        ubk, ubr = np.full(len(ub), EXTRA_UB[0]), np.full(len(ub), EXTRA_UB[1])
        ik, ip = np.full(len(s.impropers), EXTRA_IMPR[0]), np.full(len(s.impropers), math.radians(EXTRA_IMPR[1]))
        c, o = tid["CTU"], tid["OT"]
        eps4[c, o] = eps4[o, c] = 4.0 * EXTRA_NBFIX[0]
        sig2[c, o] = sig2[o, c] = (EXTRA_NBFIX[1] / 2 ** (1.0 / 6.0)) ** 2
        e14 = eps.copy()
        r14 = rmh.copy()
        e14[c], r14[c] = EXTRA_14
        sh14 = r14 / 2 ** (1.0 / 6.0)
        eps4_14 = 4.0 * np.sqrt(np.outer(e14, e14))
        sig2_14 = (sh14[:, None] + sh14[None, :]) ** 2
    cons = [(a, b) for a, b in s.bonds if s.mass[a] <= 1.5 or s.mass[b] <= 1.5]
    cd = []
    for a, b in cons:
        cd.append(WATER_HH[1] if (s.types[a], s.types[b]) == ("HT", "HT") else ROH)
    return dict(n=s.n, q=s.charge.astype(float), mass=s.mass.astype(float), type=typ, ntypes=nt,
                eps4=eps4, sig2=sig2, eps4_14=eps4_14, sig2_14=sig2_14,
                bond=s.bonds.astype(np.int32), bond_k=bk, bond_r0=br,
                angle=s.angles.astype(np.int32), angle_k=ak, angle_t0=at,
                ub=ub, ub_k=ubk, ub_r0=ubr,
                dihe=dihe.astype(np.int32), dihe_k=dk, dihe_n=dn.astype(np.int32), dihe_d=dd,
                impr=s.impropers.astype(np.int32), impr_k=ik, impr_p0=ip,
                cons=np.array(cons, np.int32).reshape(-1, 2), cons_d=np.array(cd, float),
                box=s.box.astype(float), rc=s.rc, ron=s.ron, beta=s.beta, K=np.array(s.kgrid, np.int32))


# ------------------------------------------------------------------ writers
def write(s: System, outdir: str, prefix: str | None = None, extra_in: str = "") -> str:
    """Write <prefix>.crd/.psf/.prm/.rtf and fenzi.in; returns the .in path."""
    os.makedirs(outdir, exist_ok=True)
    prefix = prefix or s.name
    crd, psf, prm, rtf = (prefix + x for x in (".crd", ".psf", ".prm", ".rtf"))
    n = s.n
    with open(os.path.join(outdir, rtf), "w") as f:
        f.write("* synthetic topology (type masses)\n*\n   36  1\n\n")
        for t, i in sorted(RTF_IDS.items(), key=lambda kv: kv[1]):
            f.write(f"MASS   {i:3d} {t:<6s} {TYPES[t][0]:10.5f} X ! synthetic\n")
        f.write("\nEND\n")
    with open(os.path.join(outdir, prm), "w") as f:
        f.write("* synthetic parameters\n*\n\nBONDS\n")
        f.write(f"OT   HT   {WATER_BOND[0]:8.3f} {WATER_BOND[1]:8.4f}\n")
        f.write(f"HT   HT   {WATER_HH[0]:8.3f} {WATER_HH[1]:8.4f}\n")
        f.write(f"CTU  CTU  {CHAIN_BOND[0]:8.3f} {CHAIN_BOND[1]:8.4f}\n")
        f.write("\nANGLES\n")
        f.write(f"HT   OT   HT   {WATER_ANGLE[0]:8.3f} {WATER_ANGLE[1]:8.3f}\n")
        ub = f" {EXTRA_UB[0]:8.3f} {EXTRA_UB[1]:8.4f}" if s.extras else ""
        f.write(f"CTU  CTU  CTU  {CHAIN_ANGLE[0]:8.3f} {CHAIN_ANGLE[1]:8.3f}{ub}\n")
        f.write("\nDIHEDRALS\n")
        f.write(f"CTU  CTU  CTU  CTU  {CHAIN_DIHE[0]:8.4f} {CHAIN_DIHE[1]:d} {CHAIN_DIHE[2]:8.2f}\n")
        if s.extras:
            f.write(f"CTU  CTU  CTU  CTU  {EXTRA_DIHE2[0]:8.4f} {EXTRA_DIHE2[1]:d} {EXTRA_DIHE2[2]:8.2f}\n")
        f.write("\nIMPROPER\n")
        if s.extras:
            f.write(f"CTU  X    X    CTU  {EXTRA_IMPR[0]:8.4f} 0 {EXTRA_IMPR[1]:8.2f}\n")
        f.write("\n")
        f.write("NONBONDED nbxmod  5 atom cdiel shift vatom vdistance vswitch -\n")
        f.write("cutnb 14.0 ctofnb 12.0 ctonnb 10.0 eps 1.0 e14fac 1.0 wmin 1.5\n\n")
        for t in ("OT", "HT", "CTU"):
            x14 = f"   0.0 {-EXTRA_14[0]:10.4f} {EXTRA_14[1]:10.4f}" if (s.extras and t == "CTU") else ""
            f.write(f"{t:<5s} 0.0  {-TYPES[t][1]:10.4f} {TYPES[t][2]:10.4f}{x14}\n")
        f.write("\nNBFIX\n")
        if s.extras:
            f.write(f"CTU  OT  {-EXTRA_NBFIX[0]:10.4f} {EXTRA_NBFIX[1]:10.4f}\n")
        f.write("\nEND\n")
    with open(os.path.join(outdir, crd), "w") as f:
        f.write("* synthetic coordinates\n*\n")
        ext = n > 99999
        f.write(f"{n:10d}  EXT\n" if ext else f"{n:5d}\n")
        for i in range(n):
            x, y, z = s.pos[i]
            if ext:
                f.write(f"{i + 1:10d}{s.resids[i]:10d}  {s.resnames[i]:<8s}  {s.atom_names[i]:<8s}"
                        f"{x:20.10f}{y:20.10f}{z:20.10f}  {s.segids[i]:<8s}  {s.resids[i]:<8d}{0.0:20.10f}\n")
            else:
                f.write(f"{i + 1:5d}{s.resids[i]:5d} {s.resnames[i]:<4s} {s.atom_names[i]:<4s}"
                        f"{x:10.5f}{y:10.5f}{z:10.5f} {s.segids[i]:<4s} {s.resids[i]:<4d}{0.0:10.5f}\n")
    with open(os.path.join(outdir, psf), "w") as f:
        f.write("PSF EXT\n\n       1 !NTITLE\n* synthetic structure\n\n")
        f.write(f"{n:10d} !NATOM\n")
        for i in range(n):
            t = s.types[i]
            f.write(f"{i + 1:10d} {s.segids[i]:<8s} {s.resids[i]:<8d} {s.resnames[i]:<8s} {s.atom_names[i]:<8s} "
                    f"{RTF_IDS[t]:4d} {s.charge[i]:14.6f}{s.mass[i]:14.4f}           0\n")

        def section(arr, width, tag):
            f.write(f"\n{len(arr):10d} !{tag}\n")
            flat = (np.asarray(arr, np.int64) + 1).reshape(-1)
            per = width
            for k in range(0, len(flat), per):
                f.write("".join(f"{v:10d}" for v in flat[k:k + per]) + "\n")

        section(s.bonds, 8, "NBOND: bonds")
        section(s.angles, 9, "NTHETA: angles")
        section(s.dihedrals, 8, "NPHI: dihedrals")
        section(s.impropers, 8, "NIMPHI: impropers")
        f.write(f"\n{0:10d} !NDON: donors\n\n\n{0:10d} !NACC: acceptors\n\n\n{0:10d} !NNB\n\n")
        f.write(f"{1:10d}{0:10d} !NGRP NST2\n{0:10d}{0:10d}{0:10d}\n\n")
    inpath = os.path.join(outdir, "fenzi.in")
    with open(inpath, "w") as f:
        f.write(f"# synthetic {s.name}: {n} atoms\n")
        f.write(f"coordinates {crd}\nstructure {psf}\nparameters {prm}\ntopology {rtf}\n")
        f.write(f"seed {s.seed}\ntemperature {s.temperature}\ntimestep {s.timestep}\n")
        f.write("startstep 0\ndynasteps 1000\noutputTiming 100\n")
        f.write(f"cuton {s.ron}\ncutoff {s.rc}\npairlistdist {s.pairlist}\n")
        f.write(f"cellBasisVector1 {s.box[0]} 0.0 0.0\ncellBasisVector2 0.0 {s.box[1]} 0.0\n"
                f"cellBasisVector3 0.0 0.0 {s.box[2]}\n")
        f.write(f"PMEGridSizeX {s.kgrid[0]}\nPMEGridSizeY {s.kgrid[1]}\nPMEGridSizeZ {s.kgrid[2]}\n")
        f.write(f"KAPPa {s.beta}\nshake on {s.shake_tol:g}\n")
        f.write(extra_in)
    return inpath


def ensemble_sizes(nsys=256, seed=2345, nw_min=216, nw_max=2000):
    """Waters per box of ensemble(): uniform in [nw_min, nw_max], seeded."""
    return np.random.default_rng(seed).integers(nw_min, nw_max + 1, size=nsys)


def ensemble(nsys=256, seed=2345, nw_min=216, nw_max=2000, rc=9.0, ron=7.5, only=None):
    """Independent TIP3P boxes (sizes uniform in [nw_min, nw_max] waters, seeded), each
    at 0.0334 waters/A^3 with its own PME grid: smallest 2^a 3^b 5^c >= L / 1.2.
    only: indices of the boxes to build (a shard); box i is the same in every shard."""
    sizes = ensemble_sizes(nsys, seed, nw_min, nw_max)
    out = []
    for i, nw in enumerate(sizes):
        if only is not None and i not in only:
            continue
        L = (nw / 0.0334) ** (1.0 / 3.0)
        out.append(build(name=f"box{i:03d}", nw=int(nw), box=L, kgrid=fft_friendly(L / 1.2), rc=rc, ron=ron,
                         seed=seed + 1 + i))
    return out
