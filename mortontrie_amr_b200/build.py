"""Build libmtlbm.so (sm_100a) in-tree with nvcc.

The FP64 translation units (multi-level path, the FP64 dense kernel and the
lattice classification, whose wall distances must equal the host mesher's)
are compiled with --fmad=false so that their arithmetic keeps the reference's
rounding; the reduced-precision dense kernels use FMA.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmtlbm.so")
OBJ = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
                 "--expt-relaxed-constexpr"]
SOURCES = {
    "mt_capi.cu": [],
    "mt_amr.cu": [],
    "mt_amr_f64.cu": ["--fmad=false"],
    "mt_amr_lp.cu": [],
    "mt_dense_f64.cu": ["--fmad=false"],
    "mt_dense_lp.cu": [],
    "mt_mesh.cu": ["--fmad=false"],
}


def _deps():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    out.append(os.path.join(ROOT, "include", "mt_lbm.h"))
    out.append(os.path.abspath(__file__))
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ, exist_ok=True)

    def comp(item):
        src, extra = item
        obj = os.path.join(OBJ, src.replace(".cu", ".o"))
        cmd = [NVCC] + COMMON + extra + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", os.path.join(CSRC, src),
                                                                                     "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr[-6000:]}")
        if verbose or ptxas_info:
            sys.stderr.write(r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(comp, SOURCES.items()))
    tmp = LIB + ".tmp"
    subprocess.run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
