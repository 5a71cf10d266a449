"""Generates tests/golden/dmpc_small.json from the reference's own example deck
tests/examples_fenzi/dmpc_small (the only complete input set the reference ships).

Every number here is computed from the raw files by this script alone (no product
code): the PSF section headers, and an independent restatement of the exclusion /
1-4 / SHAKE-constraint rules (src/prmread.cu:1757-1761, 2928-3062) over the PSF lists.
Run: python tests/golden/make_dmpc_small.py [reference_root]   (default $FENZI_REFERENCE)
"""
import json
import os
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FENZI_REFERENCE", "")
if not REF:
    sys.exit("give the reference root as the argument or in $FENZI_REFERENCE")
DECK = os.path.join(REF, "tests", "examples_fenzi", "dmpc_small")


def section(lines, tag):
    for k, ln in enumerate(lines):
        if tag in ln:
            return int(ln.split()[0]), k
    raise KeyError(tag)


def ints_after(lines, k, count, per):
    vals = []
    j = k + 1
    while len(vals) < count * per:
        vals += [int(x) - 1 for x in lines[j].split()]
        j += 1
    return [tuple(vals[i:i + per]) for i in range(0, count * per, per)]


def main():
    lines = open(os.path.join(DECK, "dmpc_small.psf")).read().splitlines()
    natom, ka = section(lines, "!NATOM")
    q, mass = [], []
    for ln in lines[ka + 1:ka + 1 + natom]:
        t = ln.split()
        q.append(float(t[6]))
        mass.append(float(t[7]))
    nb, kb = section(lines, "!NBOND")
    nt, kt = section(lines, "!NTHETA")
    nphi, kp = section(lines, "!NPHI")
    nimp, _ = section(lines, "!NIMPHI")
    bonds = ints_after(lines, kb, nb, 2)
    angles = ints_after(lines, kt, nt, 3)
    dihes = ints_after(lines, kp, nphi, 4)
    key = lambda a, b: (min(a, b), max(a, b))
    ew = {key(a, b) for a, b in bonds if a != b} | {key(a, c) for a, b, c in angles if a != c}
    p14 = {key(a, d) for a, b, c, d in dihes if a != d} - ew
    cons = [(a, b) for a, b in bonds if mass[a] <= 1.5 or mass[b] <= 1.5]
    parent = list(range(natom))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in cons:
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)
    clusters = {find(a) for a, _ in cons}
    crd = open(os.path.join(DECK, "dmpc_small.crd")).read().splitlines()
    ncrd = int([ln for ln in crd if not ln.startswith("*")][0].split()[0])
    out = dict(natom=natom, ncrd=ncrd, nbond=nb, nangle=nt, ndihedral=nphi, nimproper=nimp,
               nexcl_pairs=len(ew), n14_pairs=len(p14), nconstraint=len(cons), ncluster=len(clusters),
               net_charge=round(sum(q), 6), total_mass=round(sum(mass), 4),
               box=[46.8, 46.8, 76.0], pme_grid=[64, 64, 64], kappa=0.32, cutoff=8.0, cuton=7.0,
               pairlistdist=9.5, shake_tol=1e-10, seed=2345, temp_reset_every=20000)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dmpc_small.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(dst, out)


if __name__ == "__main__":
    main()
