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


def _c_layout(struct, fields, tmp_path):
    """sizeof and offsetof of a header struct, from a C program built with gcc."""
    import subprocess
    src = tmp_path / "layout.c"
    body = "".join(f'    printf("%zu\\n", offsetof({struct}, {f}));\n' for f in fields)
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "mt_lbm.h"\nint main(void) {\n'
                   f'    printf("%zu\\n", sizeof({struct}));\n{body}    return 0;\n}}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    return [int(v) for v in out]


def test_ctypes_structs_match_header_layout(tmp_path):
    from mortontrie_amr_b200.lbm import mt_case_desc, mt_mesh_spec
    for cls, name in ((mt_case_desc, "mt_case_desc"), (mt_mesh_spec, "mt_mesh_spec")):
        fields = [f for f, _ in cls._fields_]
        got = _c_layout(name, fields, tmp_path)
        want = [ctypes.sizeof(cls)] + [getattr(cls, f).offset for f in fields]
        assert got == want, (name, got, want)


def test_storage_shift_levels():
    """storage_shift options map to one velocity per level in mt_case_desc."""
    import numpy as np
    import pytest
    from mortontrie_amr_b200.case import nested_sphere_case
    from mortontrie_amr_b200.lbm import MAX_LEVELS, make_desc, storage_shift_of
    case = nested_sphere_case(coarse=(48, 24, 24), max_level=2, center=(16, 12, 12), radius=2.0,
                              half_widths=(4.0, 2.5), re=50.0, mesh="device")
    ubc = tuple(float(v) for v in case.params.u_bc)
    z = (0.0, 0.0, 0.0)
    assert storage_shift_of(case, None) == [z] * 3
    assert storage_shift_of(case, "inlet") == [ubc] * 3
    assert storage_shift_of(case, "far_field") == [ubc, ubc, z]
    assert storage_shift_of(case, (0.01, 0.02, 0.03)) == [(0.01, 0.02, 0.03)] * 3
    per = [(0.01, 0, 0), (0, 0.02, 0), (0, 0, 0.03)]
    assert storage_shift_of(case, per) == [tuple(float(v) for v in r) for r in per]
    with pytest.raises(ValueError):
        storage_shift_of(case, "outlet")
    with pytest.raises(ValueError):
        storage_shift_of(case, [(0, 0, 0)] * 2)
    d = make_desc(case, "f16", "far_field")
    got = np.array([[d.u_shift[l][a] for a in range(3)] for l in range(MAX_LEVELS)])
    want = np.zeros((MAX_LEVELS, 3))
    want[:2] = ubc
    assert np.array_equal(got, want)
