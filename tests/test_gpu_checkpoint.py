"""Restart files in the reference's binary and ascii layouts (SaveCheckpointBinary/Ascii,
LoadCheckpointBinary/Ascii): header and records as the reference writes them, exact
round trip for binary, 1e-6 for the ascii %10f columns, and a restarted run that
follows the uninterrupted one."""
import os
import struct
import tempfile

import numpy as np
import pytest

import fenzi_b200 as fz
from tests.helpers import system

pytestmark = pytest.mark.gpu


def _sys():
    _, path = system("small")
    s = fz.FenZi.ReadInput(path).LoadSystem()
    s.InitMem(0)
    return s


def test_binary_layout_and_round_trip():
    s = _sys()
    s.InitVelocity(T=300.0, seed=3, counter=0)
    s.SingleStep(30)
    d = tempfile.mkdtemp(prefix="fzck_")
    fb = os.path.join(d, "x.rst")
    s.SaveCheckpoint(fb, "b")
    raw = open(fb, "rb").read()
    n, step = struct.unpack_from("<ii", raw, 0)
    seed, = struct.unpack_from("<d", raw, 8)
    box = struct.unpack_from("<3f", raw, 16)
    bvel = struct.unpack_from("<3f", raw, 28)
    rec = np.frombuffer(raw, dtype="<f4", offset=40).reshape(n, 6)
    assert n == s.n and step == 30 and len(raw) == 40 + 24 * n
    assert seed == float(s.cfg.seed) and np.allclose(box, s.cfg.box[:3]) and bvel == (0.0, 0.0, 0.0)
    assert np.array_equal(rec[:, :3], s.positions().astype(np.float32))
    assert np.array_equal(rec[:, 3:], s.velocities().astype(np.float32))
    fa = os.path.join(d, "x.rsta")
    s.SaveCheckpoint(fa, "a")
    t = _sys()
    t.LoadCheckpoint(fb, "b")
    assert np.array_equal(t.positions(), s.positions()) and np.array_equal(t.velocities(), s.velocities())
    u = _sys()
    u.LoadCheckpoint(fa, "a")
    assert np.abs(u.positions() - s.positions()).max() <= 1e-6
    assert np.abs(u.velocities() - s.velocities()).max() <= 1e-6
    # a restarted run follows the uninterrupted one
    s.SingleStep(20)
    t.SingleStep(20)
    assert np.abs(t.positions() - s.positions()).max() < 1e-3
    assert t.EvalProps()["step"] == s.EvalProps()["step"] == 50
    for x in (s, t, u):
        x.close()


def test_load_rejects_wrong_atom_count_and_missing_file():
    s = _sys()
    d = tempfile.mkdtemp(prefix="fzck_")
    bad = os.path.join(d, "bad.rst")
    with open(bad, "wb") as f:
        f.write(struct.pack("<iid3f3f", s.n + 1, 0, 1.0, 1, 1, 1, 0, 0, 0))
    with pytest.raises(fz.FenZiError) as ei:
        s.LoadCheckpoint(bad, "b")
    assert ei.value.code == 2  # FZ_ERR_PARSE
    with pytest.raises(fz.FenZiError) as ei:
        s.LoadCheckpoint(os.path.join(d, "missing.rst"), "b")
    assert ei.value.code == 1  # FZ_ERR_IO
    s.close()


def _records(raw):
    out, o = [], 0
    while o < len(raw):
        n, = struct.unpack_from("<i", raw, o)
        out.append(raw[o + 4:o + 4 + n])
        assert struct.unpack_from("<i", raw, o + 4 + n)[0] == n
        o += 8 + n
    return out


def test_dcd_layout_and_frames():
    s = _sys()
    s.InitVelocity(T=300.0, seed=5, counter=0)
    path = os.path.join(tempfile.mkdtemp(prefix="fzdcd_"), "t.dcd")
    frames = []
    with fz.Trajectory(s, path, every=10) as tr:
        for _ in range(3):
            s.SingleStep(10)
            tr.write()
            frames.append(s.positions().astype(np.float32))
    r = _records(open(path, "rb").read())
    assert r[0][:4] == b"CORD"
    ctl = struct.unpack("<20i", r[0][4:84])
    assert ctl[0] == 3 and ctl[1] == 10 and ctl[2] == 10 and ctl[3] == 30 and ctl[10] == 1 and ctl[19] == 34
    assert abs(struct.unpack("<f", r[0][40:44])[0] - s.cfg.timestep_ps / 4.888821e-2) < 1e-6
    assert struct.unpack_from("<i", r[1])[0] == 1 and len(r[1]) == 84
    assert struct.unpack("<i", r[2])[0] == s.n
    assert len(r) == 3 + 3 * 4
    for k in range(3):
        cell = struct.unpack("<6d", r[3 + 4 * k])
        assert np.allclose([cell[0], cell[2], cell[5]], s.cfg.box[:3]) and cell[1] == cell[3] == cell[4] == 0.0
        xyz = np.stack([np.frombuffer(r[4 + 4 * k + c], dtype="<f4") for c in range(3)], axis=1)
        assert np.array_equal(xyz, frames[k])
    s.close()
