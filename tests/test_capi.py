"""The C-ABI library loads and exports every entry point include/mt_lbm.h
declares (no device work: this runs without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "mt_lbm.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(mt_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = _declared()
    assert "mt_step" in names and "mt_case_build" in names and len(names) >= 30


def test_library_exports_every_declared_symbol():
    from mortontrie_amr_b200 import build as B
    B.build()
    lib = ctypes.CDLL(B.LIB)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from mortontrie_amr_b200.lbm import EXPORTS
    assert sorted(EXPORTS) == _declared()
