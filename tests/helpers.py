"""Shared helpers of the test suite (golden loading, oracle runs)."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TAG_BC = 32


def load_golden(name):
    from golden_cases import build_case
    z = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    spec = meta["spec"]
    case = build_case(spec)
    return spec, case, z, meta


def sha(a) -> bytes:
    return hashlib.sha256(np.ascontiguousarray(a, np.float64).tobytes()).digest()


def init_of(case, spec):
    from mortontrie_amr_b200.case import perturbed_populations
    return perturbed_populations(case, seed=spec["seed"]) if spec["init"] == "perturbed" else None


def run_oracle(case, steps, init=None):
    import oracle as O
    oc = O.OracleCase(case)
    if init is not None:
        for l, (_, f) in enumerate(init):
            oc.set_populations(l, f)
    oc.step(steps)
    return oc


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
