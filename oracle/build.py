"""Build recipe for the test oracle and the reference harness.

TEST INFRASTRUCTURE ONLY.

* ``libmt_oracle.so`` -- the C restatement in ``mt_oracle.c`` (FP64, no FMA
  contraction, like the reference built with g++ on x86-64).
* ``_ref/refharness_q{Q}_l{L}`` -- the reference's own LBM translation units
  compiled from where they lie in the reference checkout, linked with
  ``refharness/harness.cpp``.  Two things shadow reference headers, found
  first through ``-I-`` (which turns off the "directory of the including
  file first" rule for quoted includes):

    1. ``refharness/Constants.h`` replaces ``header/Constants.h`` (the
       reference keeps its case configuration in compile-time constants);
    2. ``_ref/shim_q{Q}_l{L}/LBM_Manager.hpp`` is written here from
       ``header/LBM_Manager.hpp`` with one edit: the counters declared at
       ``LBM_Manager.hpp:103-104`` as ``std::array<uint, C_max_level+1>
       run_col_times{0,0,0}`` get an empty initialiser, because three
       initialisers do not compile unless C_max_level == 2.

  Nothing else in the reference is changed.  The reference's own Makefile is
  not used (it links HDF5, which this image lacks); the flags are its
  ``-std=c++17 -O3`` (Makefile:15-17).  Outputs go to ``oracle/_ref`` only.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REF = "/root/reference"
REF_TUS = [
    "LBM_Manager.cpp",
    "LBM_Simulator.cpp",
    "lbm_kernel/Collision_Manager.cpp",
    "lbm_kernel/Collision_Cumulant.cpp",
    "lbm_kernel/Stream_Manager.cpp",
    "BC/D3Q19_BC_Manager.cpp",
    "BC/NonEquilibrumExtrapolation.cpp",
    "ComplexBoundary_Manager.cpp",
    "Morton_Assist.cpp",
]
HARNESS_VARIANTS = [(19, 0), (19, 1), (19, 2), (27, 0), (27, 1), (27, 2)]


def oracle_lib_path() -> str:
    return os.path.join(HERE, "libmt_oracle.so")


def build_oracle_lib(force: bool = False) -> str:
    out = oracle_lib_path()
    src = os.path.join(HERE, "mt_oracle.c")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    subprocess.run(["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                    "-Wall", "-o", out, src, "-lm"], check=True)
    return out


def harness_path(q: int, L: int) -> str:
    return os.path.join(HERE, "_ref", f"refharness_q{q}_l{L}")


def _shim_header(q: int, L: int) -> str:
    d = os.path.join(HERE, "_ref", f"shim_q{q}_l{L}")
    os.makedirs(d, exist_ok=True)
    src = open(os.path.join(REF, "header", "LBM_Manager.hpp")).read()
    old_col = "run_col_times{0,0,0};"
    old_stm = "run_stm_times{0,0,0};"
    if old_col not in src or old_stm not in src:
        raise RuntimeError("LBM_Manager.hpp no longer has the expected counter initialisers")
    src = src.replace(old_col, "run_col_times{};").replace(old_stm, "run_stm_times{};")
    with open(os.path.join(d, "LBM_Manager.hpp"), "w") as fh:
        fh.write(src)
    return d


def build_refharness(q: int, L: int, force: bool = False) -> str:
    out = harness_path(q, L)
    if not os.path.isdir(REF):
        if os.path.exists(out):
            return out
        raise FileNotFoundError("reference checkout not present and no prebuilt harness")
    deps = [os.path.join(HERE, "refharness", "harness.cpp"), os.path.join(HERE, "refharness", "Constants.h"),
            os.path.abspath(__file__)]
    if not force and os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(p) for p in deps):
        return out
    shim = _shim_header(q, L)
    objdir = os.path.join(HERE, "_ref", f"obj_q{q}_l{L}")
    os.makedirs(objdir, exist_ok=True)
    # with -I- every directory reached by a quoted include must be listed,
    # including the one libstdc++'s parallel-algorithm headers use
    gxx = subprocess.run(["g++", "-dumpversion"], capture_output=True, text=True).stdout.strip()
    inc = ["-I", shim, "-I", os.path.join(HERE, "refharness"), "-I", os.path.join(REF, "header"),
           "-I", os.path.join(REF, "header", "lbm_kernel"), "-I", os.path.join(REF, "header", "BC"), "-I", REF,
           "-I", f"/usr/include/c++/{gxx}/pstl", "-I-"]
    flags = ["g++", "-std=c++17", "-O3", "-w", f"-DHC_Q={q}", f"-DHC_L={L}"] + inc
    srcs = [os.path.join(REF, t) for t in REF_TUS] + [os.path.join(HERE, "refharness", "harness.cpp")]

    def comp(src):
        obj = os.path.join(objdir, os.path.basename(src).replace(".cpp", ".o"))
        r = subprocess.run(flags + ["-c", src, "-o", obj], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile {src} failed:\n{r.stderr[-4000:]}")
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(comp, srcs))
    subprocess.run(["g++", "-o", out] + objs, check=True)
    return out


def build_all(harness: bool = True) -> None:
    build_oracle_lib()
    if harness and os.path.isdir(REF):
        for q, L in HARNESS_VARIANTS:
            build_refharness(q, L)


if __name__ == "__main__":
    build_all(harness="--no-harness" not in sys.argv)
