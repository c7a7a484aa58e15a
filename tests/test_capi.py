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
