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

  The periodic variants (``_ref/refharness_q{Q}_l{L}_periodic``) add a third:
  ``_ref/shim_q{Q}_l{L}_periodic/Morton_Assist.h``, written from
  ``header/Morton_Assist.h`` with the result of ``find_neighbor``
  (``Morton_Assist.h:254-280``) passed through a wrap of the level-0 box on
  the axes the harness input marks periodic.  The reference has no periodic
  path that builds (``BC/Periodic.cpp`` needs the ghost layers that
  ``BC_NO_GHOST`` removes), and every neighbour lookup of the step (stream,
  boundary, IB) goes through ``find_neighbor``; the explosion and coalescence
  children (``find_x1``/``find_y1``/``find_z1`` inside one parent) never
  cross the box.  With no axis marked the wrap returns the reference's key.

  Nothing else in the reference is changed.  The reference's own Makefile is
  not used (it links HDF5, which this image lacks); the flags are its
  ``-std=c++17 -O3`` (Makefile:15-17).  Outputs go to ``oracle/_ref`` only.

The reference checkout is read from ``$MT_REFERENCE_DIR`` (default
``/root/reference``); without it the prebuilt harnesses under ``_ref`` are
used as they are.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("MT_REFERENCE_DIR", "/root/reference")
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
    "tecplot.cpp",
    "Lat_Voxelize.cpp",
    "Shape.cpp",
]
HARNESS_VARIANTS = [(19, 0), (19, 1), (19, 2), (19, 3), (27, 0), (27, 1), (27, 2), (27, 3)]
# (Q, L) of the harnesses built with the periodic find_neighbor wrap
PERIODIC_VARIANTS = [(19, 1), (27, 1)]


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


def harness_path(q: int, L: int, periodic: bool = False) -> str:
    return os.path.join(HERE, "_ref", f"refharness_q{q}_l{L}" + ("_periodic" if periodic else ""))


_WRAP = r"""
/* ---- inserted by oracle/build.py: periodic wrap of the level-0 box ---- */
inline int hc_periodic[3] = {0, 0, 0};
inline long long hc_extent0[3] = {0, 0, 0};
inline unsigned long long hc_dilate(unsigned long long v)
{
    v &= 0x1FFFFFULL;
    v = (v | (v << 32)) & 0x1F00000000FFFFULL;
    v = (v | (v << 16)) & 0x1F0000FF0000FFULL;
    v = (v | (v << 8)) & 0x100F00F00F00F00FULL;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ULL;
    v = (v | (v << 2)) & 0x1249249249249249ULL;
    return v;
}
inline unsigned long long hc_compact(unsigned long long v)
{
    v &= 0x1249249249249249ULL;
    v = (v ^ (v >> 2)) & 0x10C30C30C30C30C3ULL;
    v = (v ^ (v >> 4)) & 0x100F00F00F00F00FULL;
    v = (v ^ (v >> 8)) & 0x1F0000FF0000FFULL;
    v = (v ^ (v >> 16)) & 0x1F00000000FFFFULL;
    v = (v ^ (v >> 32)) & 0x1FFFFFULL;
    return v;
}
/* key: the cell; rst: find_neighbor's result for the shift (sx, sy, sz) at
 * `level`.  On a periodic axis whose shifted coordinate leaves [0, n_l)
 * (n_l = level-0 extent << level) the axis bits of rst are replaced by the
 * wrapped coordinate. */
inline D_morton hc_periodic_wrap(const D_morton &key, const D_morton &rst, unsigned level, int sx, int sy, int sz)
{
    const int s[3] = {sx, sy, sz};
    unsigned long long k = key.to_ullong(), r = rst.to_ullong();
    const unsigned sh = C_max_level - level;
    for (int a = 0; a < 3; ++a) {
        if (!hc_periodic[a] || s[a] == 0) continue;
        long long n = hc_extent0[a] << level;
        long long t = (long long)(hc_compact(k >> a) >> sh) + s[a];
        if (t >= 0 && t < n) continue;
        t = ((t % n) + n) % n;
        unsigned long long m = 0x1249249249249249ULL << a;
        r = (r & ~m) | (hc_dilate((unsigned long long)t << sh) << a);
    }
    return D_morton(r);
}
/* ---- end of insertion ---- */
"""


def _morton_shim(d: str) -> None:
    src = open(os.path.join(REF, "header", "Morton_Assist.h")).read()
    head = "inline D_morton Morton_Assist::find_neighbor(const D_morton& key, const uint level, const int x_shift, " \
           "const int y_shift, const int z_shift)"
    i = src.find(head)
    if i < 0 or src.count(head) != 1:
        raise RuntimeError("Morton_Assist.h no longer has the expected find_neighbor definition")
    j = src.find("return rst_code;", i)
    k = src.find("\n}", i)
    if j < 0 or j > k:
        raise RuntimeError("Morton_Assist.h find_neighbor no longer ends in 'return rst_code;'")
    src = (src[:i] + _WRAP + src[i:j]
           + "return hc_periodic_wrap(key, rst_code, level, x_shift, y_shift, z_shift);" + src[j + len("return rst_code;"):])
    with open(os.path.join(d, "Morton_Assist.h"), "w") as fh:
        fh.write(src)


def _shim_header(q: int, L: int, periodic: bool = False) -> str:
    d = os.path.join(HERE, "_ref", f"shim_q{q}_l{L}" + ("_periodic" if periodic else ""))
    os.makedirs(d, exist_ok=True)
    if periodic:
        _morton_shim(d)
    src = open(os.path.join(REF, "header", "LBM_Manager.hpp")).read()
    old_col = "run_col_times{0,0,0};"
    old_stm = "run_stm_times{0,0,0};"
    if old_col not in src or old_stm not in src:
        raise RuntimeError("LBM_Manager.hpp no longer has the expected counter initialisers")
    src = src.replace(old_col, "run_col_times{};").replace(old_stm, "run_stm_times{};")
    with open(os.path.join(d, "LBM_Manager.hpp"), "w") as fh:
        fh.write(src)
    return d


def build_refharness(q: int, L: int, force: bool = False, periodic: bool = False) -> str:
    out = harness_path(q, L, periodic)
    if not os.path.isdir(REF):
        if os.path.exists(out):
            return out
        raise FileNotFoundError("reference checkout not present and no prebuilt harness")
    deps = [os.path.join(HERE, "refharness", "harness.cpp"), os.path.join(HERE, "refharness", "Constants.h"),
            os.path.abspath(__file__)]
    if not force and os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(p) for p in deps):
        return out
    shim = _shim_header(q, L, periodic)
    objdir = os.path.join(HERE, "_ref", f"obj_q{q}_l{L}" + ("_periodic" if periodic else ""))
    os.makedirs(objdir, exist_ok=True)
    # with -I- every directory reached by a quoted include must be listed,
    # including the one libstdc++'s parallel-algorithm headers use
    gxx = subprocess.run(["g++", "-dumpversion"], capture_output=True, text=True).stdout.strip()
    inc = ["-I", shim, "-I", os.path.join(HERE, "refharness"), "-I", os.path.join(REF, "header"),
           "-I", os.path.join(REF, "header", "lbm_kernel"), "-I", os.path.join(REF, "header", "BC"), "-I", REF,
           "-I", f"/usr/include/c++/{gxx}/pstl", "-I-"]
    flags = ["g++", "-std=c++17", "-O3", "-w", f"-DHC_Q={q}", f"-DHC_L={L}"] + (["-DHC_PERIODIC"] if periodic else []) + inc
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
        for q, L in PERIODIC_VARIANTS:
            build_refharness(q, L, periodic=True)


if __name__ == "__main__":
    build_all(harness="--no-harness" not in sys.argv)
