"""The C-ABI library loads and exports every symbol include/fenzi_b200.h declares."""
import ctypes
import os
import re

import pytest

import fenzi_b200 as fz

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "fenzi_b200.h")


def declared():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"^\s*(?:fz_status|const char\*|void\*)\s+(fz_\w+)\s*\(", txt, re.M)))


def test_header_symbols_exported():
    names = declared()
    assert len(names) >= 20
    lib = ctypes.CDLL(fz.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(fz.EXPORTS)


def test_version_and_error_channel():
    assert b"sm_100a" in fz.lib().fz_version()
    import ctypes as C
    cfg = fz.Config()
    rc = fz.lib().fz_read_input(b"/nonexistent/x.in", C.byref(cfg))
    assert rc == 1 and "not found" in fz.last_error()


def test_device_calls_before_upload_fail_cleanly():
    from tests.helpers import system
    _, path = system("small")
    s = fz.FenZi.ReadInput(path).LoadSystem()
    for call in (lambda: s.SingleStep(1), lambda: s.SaveCheckpoint("/nonexistent/x.rst", "b"),
                 lambda: s.LoadCheckpoint("/nonexistent/x.rst", "b")):
        with pytest.raises(fz.FenZiError) as ei:
            call()
        assert ei.value.code == 7  # FZ_ERR_STATE


def test_server_without_gpu_fails_cleanly():
    """No device: fz_server_create returns an error status (no worker thread starts)."""
    import ctypes as C
    L = fz.lib()
    h = C.c_void_p()
    code = L.fz_server_create(0, 1e9, 10, 2, C.byref(h))
    if code == 0:  # a GPU is present: nothing to check here
        L.fz_server_free(h)
        pytest.skip("a CUDA device is present")
    assert code in (3, 6)  # FZ_ERR_CUDA / FZ_ERR_ARG
    assert fz.last_error()


def test_plain_header_symbols_exported():
    """libfenzi_plain.so (the comparator path) exports every symbol of fenzi_plain.h."""
    from fenzi_b200 import plain
    txt = open(os.path.join(os.path.dirname(HDR), "fenzi_plain.h")).read()
    names = sorted(set(re.findall(r"^\s*fz_status\s+(fz_plain_\w+)\s*\(", txt, re.M)))
    assert len(names) == 10
    L = plain.plib()
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(plain.PLAIN_EXPORTS)


def test_plain_without_gpu_fails_cleanly():
    from tests.helpers import system
    from fenzi_b200.plain import Plain
    _, path = system("tiny")
    s = fz.FenZi.ReadInput(path).LoadSystem()
    try:
        p = Plain(s, 0)
    except fz.FenZiError as e:
        assert e.code == 3 and fz.last_error()
        return
    p.close()
    pytest.skip("a CUDA device is present")
