"""The C++ drop-in layer (include/mt_lbm.hpp): map semantics on the CPU, and
a reference-style program driving the GPU path, compared with the oracle."""
import os
import subprocess

import numpy as np
import pytest
from helpers import run_oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")


def _compile(src, out, link=False):
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), os.path.join(CPP, src), "-o", out]
    if link:
        from mortontrie_amr_b200 import build as B
        B.build()
        lib_dir = os.path.dirname(B.LIB)
        cmd += [B.LIB, f"-Wl,-rpath,{lib_dir}"]
    subprocess.run(cmd, check=True)
    return out


def test_map_semantics(tmp_path):
    exe = _compile("dmap_test.cpp", str(tmp_path / "dmap_test"))
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def test_storage_shift_table(tmp_path):
    """The per-level storage shift table built on the host (make_shift)."""
    exe = _compile("shift_test.cpp", str(tmp_path / "shift_test"))
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def test_demo_links(tmp_path):
    _compile("shim_demo.cpp", str(tmp_path / "shim_demo"), link=True)


@pytest.mark.gpu
def test_demo_matches_oracle(tmp_path):
    import oracle as O
    from golden_cases import GOLDEN_CASES, build_case
    spec = GOLDEN_CASES["sphere_q19_fh_refinit"]
    case = build_case(spec)
    exe = _compile("shim_demo.cpp", str(tmp_path / "shim_demo"), link=True)
    sets = tmp_path / "sets.bin"
    sets.write_bytes(O.harness_input(case, spec["steps"]))
    out = tmp_path / "out.bin"
    taus = [repr(t) for t in case.params.taus(case.max_level)]
    subprocess.run([exe, str(sets), str(out), str(spec["steps"])] + taus, check=True)
    data = out.read_bytes()
    oc = run_oracle(case, spec["steps"])
    off = 0
    for l in range(case.max_level + 1):
        n = int(np.frombuffer(data, np.int64, 1, off)[0])
        off += 8
        f = np.frombuffer(data, np.float64, n, off).reshape(case.q, -1)
        off += 8 * n
        g = oc.get(l)
        keep = (g["tags"] & 32) == 0
        assert np.array_equal(f[:, keep], g["f"][:, keep]), l
