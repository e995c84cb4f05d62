"""The C-ABI library loads and exports every symbol include/lightsim2grid_b200.h declares."""
import os
import re

from conftest import ROOT


def _declared():
    txt = open(os.path.join(ROOT, "include", "lightsim2grid_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pf_[A-Za-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = _declared()
    for must in ("pf_plan_create", "pf_solve", "pf_batch_n1", "pf_batch_ts", "pf_get_J", "pf_timers",
                 "pf_plan_destroy", "pf_batch_device"):
        assert must in names


def test_library_exports_all_declared_symbols():
    import ctypes
    from lightsim2grid_b200 import build, _native

    build.build()
    lib = ctypes.CDLL(build.LIB)
    for name in _declared():
        assert hasattr(lib, name), name
    assert set(_native.SYMBOLS) == set(_declared())
    _native.load()


def test_missing_library_fails_loudly(tmp_path):
    import pytest
    from lightsim2grid_b200 import _native

    with pytest.raises(ImportError):
        _native.load(str(tmp_path / "nope.so"))



def test_n1_order_rejects_null_arguments():
    """pf_n1_order validates its arguments before touching a plan (no GPU needed)."""
    from lightsim2grid_b200 import _native as nat

    lib = nat.load()
    assert lib.pf_n1_order(None, 0, None, None, None, None, None) != 0
