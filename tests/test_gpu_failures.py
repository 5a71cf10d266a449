"""Failure paths of the step, made on the host: each ends in a status code and a message
from fz_step, with no fault, trap or hang on the GPU.

- SHAKE / SETTLE on a constraint set with no solution (an H-H constraint longer than
  the two O-H constraints together): the reference's SHAKE loop has no iteration cap
  (src/shake.cu:195-271); here the Newton solve stops at its cap and SETTLE at its
  first impossible square root, both raise the status word, and fz_step returns
  FZ_ERR_SHAKE.  Every kernel after the failed solve stays in bounds with the
  non-finite or unconstrained coordinates it leaves (grid and cell indices are
  clamped and wrapped).
- Pair-list capacity: FZ_LIST_CAP shrinks the per-block list capacity after set-up,
  so the next rebuild overflows it; the kernels keep the entries that fit and raise
  the status word, and fz_step returns FZ_ERR_CAPACITY (src/dynamics.cu:114-118 exits
  the process instead).
"""
import os

import pytest

import fenzi_b200 as fz
from fenzi_b200 import gen_system

pytestmark = pytest.mark.gpu


def _impossible_water_box(tmp):
    s = gen_system.build(name="custom", nw=216, seed=11, rc=7.0, ron=6.0)
    path = gen_system.write(s, str(tmp))
    prm = next(os.path.join(str(tmp), f) for f in os.listdir(str(tmp)) if f.endswith(".prm"))
    text = open(prm).read()
    hh = next(ln for ln in text.splitlines() if ln.startswith("HT   HT"))
    text = text.replace(hh, "HT   HT      0.000   5.0000")  # > 2 x 0.9572: no solution
    open(prm, "w").write(text)
    return path


@pytest.mark.parametrize("settle", ["1", "0"], ids=["settle", "newton"])
def test_unsolvable_constraints_return_shake_error(tmp_path, monkeypatch, settle):
    monkeypatch.setenv("FZ_SETTLE", settle)
    s = fz.FenZi.ReadInput(_impossible_water_box(tmp_path)).LoadSystem()
    s.InitMem(0)
    s.InitVelocity(T=300.0, seed=5)
    with pytest.raises(fz.FenZiError) as err:
        s.SingleStep(3)
    assert err.value.code == 5, err.value
    assert "SHAKE did not converge" in str(err.value)
    s.close()


def test_pair_list_overflow_returns_capacity_error(monkeypatch):
    s_gen = gen_system.build(name="water3000")
    import tempfile
    path = gen_system.write(s_gen, tempfile.mkdtemp(prefix="fz_cap_"))
    monkeypatch.setenv("FZ_LIST_CAP", "64")
    s = fz.FenZi.ReadInput(path).LoadSystem()
    s.InitMem(0)  # set-up succeeds; the cap takes effect at the next rebuild
    with pytest.raises(fz.FenZiError) as err:
        s.SingleStep(2)
    assert err.value.code == 4, err.value
    assert "pair-tile capacity exceeded" in str(err.value)
    s.close()
