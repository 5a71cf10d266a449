"""Shared builders for the tests: seeded systems written through the drop-in file
formats and loaded by the product readers; the oracle is built from the generator's own
topology (gen_system.topology: every parameter resolved without the readers), so a
reader fault cannot hide in a force comparison."""
import os
import tempfile

import numpy as np

from fenzi_b200 import gen_system

_CACHE = {}
_GEN_BY_DIR = {}  # input directory -> gen_system.System written there
_TMP = tempfile.mkdtemp(prefix="fzb200_")

ORACLE_BONDED = 16 | 32 | 64 | 128 | 256 | 2 | 4  # bonds angles ub dihe impr excl p14


def system(key="small", **kw):
    """(System, in_path): cached per key."""
    if key in _CACHE:
        return _CACHE[key]
    presets = {
        "small": dict(name="custom", nw=400, nchains=2, chain_len=10, rc=8.0, ron=6.5, seed=7),
        "water3000": dict(name="water3000"),
        "large230k": dict(name="large230k", seed=2345),
        "mid": dict(name="custom", nw=8760, nchains=6, chain_len=30, box=64.0, kgrid=64, rc=10.0, ron=8.0, seed=11),
        "tiny": dict(name="custom", nw=60, nchains=1, chain_len=8, box=14.0, kgrid=16, rc=6.0, ron=5.0, seed=3),
    }
    args = dict(presets.get(key, {}))
    args.update(kw)
    s = gen_system.build(**args)
    path = gen_system.write(s, os.path.join(_TMP, key))
    _CACHE[key] = (s, path)
    _GEN_BY_DIR[os.path.realpath(os.path.dirname(path))] = s
    return s, path


def rel_rms(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def oracle_for(fz_sys, nthreads=0):
    """The oracle of a loaded system: from the generator's topology when the system
    was written by system() (reader-free), else from the product readers' topology."""
    from oracle.oracle import Oracle
    c = fz_sys.cfg
    gen = _GEN_BY_DIR.get(os.path.realpath(os.path.dirname(c.coordinates.decode())))
    if gen is None:
        return Oracle(fz_sys.topology(), nthreads=nthreads)
    topo = gen_system.topology(gen)
    # run parameters come from the configuration the system was loaded with (a test may
    # change them after reading the input file)
    topo.update(box=np.array(list(c.box)), rc=c.cutoff, ron=c.cuton, beta=c.kappa, K=np.array(list(c.pme_grid)))
    if not c.shake:
        topo.update(cons=np.zeros((0, 2), np.int32), cons_d=np.zeros(0))
    return Oracle(topo, nthreads=nthreads)
