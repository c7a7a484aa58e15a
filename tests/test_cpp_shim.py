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


def test_user_view_demo_links(tmp_path):
    _compile("user_view_demo.cpp", str(tmp_path / "user_view_demo"), link=True)


@pytest.mark.gpu
def test_user_views_match_oracle(tmp_path):
    """LBM_Manager() from the Lat_Manager singleton and config(), an
    infoPrint-shaped loop over user[l].velocity / density, and a population
    changed through user[0].df.f[q].at(code) before one more step: all
    bit-identical to the oracle doing the same."""
    import oracle as O
    from golden_cases import GOLDEN_CASES, build_case
    spec = GOLDEN_CASES["sphere_q19_fh_refinit"]
    case = build_case(spec)
    steps = 3
    exe = _compile("user_view_demo.cpp", str(tmp_path / "user_view_demo"), link=True)
    sets = tmp_path / "sets.bin"
    sets.write_bytes(O.harness_input(case, steps))
    out = tmp_path / "out.bin"
    taus = [repr(t) for t in case.params.taus(case.max_level)]
    subprocess.run([exe, str(sets), str(out), str(steps)] + taus, check=True)
    data = out.read_bytes()
    oc = run_oracle(case, steps)
    off = 0

    def take(n, dt=np.float64):
        nonlocal off
        a = np.frombuffer(data, dt, n, off)
        off += a.nbytes
        return a

    for l in range(case.max_level + 1):
        n = int(take(1, np.int64)[0])
        rho, ux, uy, uz = (take(n) for _ in range(4))
        maxv = take(1)[0]
        g = oc.get(l)
        sel = np.isin(g["keys"], case.mesh.levels[l]["lat_f"])
        assert sel.sum() == n
        assert np.array_equal(rho, g["rho"][sel]), l
        assert np.array_equal(np.stack([ux, uy, uz], axis=1), g["u"][sel]), l
        assert maxv == np.sqrt((g["u"][sel] ** 2).sum(axis=1)).max()
    key = int(take(1, np.uint64)[0])
    q = int(take(1, np.int64)[0])
    newv = take(1)[0]
    g = oc.get(0)
    i = int(np.searchsorted(g["keys"], np.uint64(key)))
    assert g["keys"][i] == key and newv == g["f"][q, i] + 1e-3
    f = g["f"].copy()
    f[q, i] = newv
    oc.set_populations(0, f, g["fcol"])
    oc.step(1)
    for l in range(case.max_level + 1):
        n = int(take(1, np.int64)[0])
        fl = take(n).reshape(case.q, -1)
        g = oc.get(l)
        keep = (g["tags"] & 32) == 0
        assert np.array_equal(fl[:, keep], g["f"][:, keep]), l
