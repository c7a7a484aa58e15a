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


def load_trace(name):
    from golden_cases import build_case
    z = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    return meta["spec"], build_case(meta["spec"]), z, meta


def trace_mismatches(case, z, d, level_state):
    """Compare one dump of a trace golden with a state: level_state(l) gives
    dict(keys, tags, f (Q, n), fcol (Q, n), rho (n,), u (3, n)) of level l.
    Returns the list of differences (empty when everything is bit-exact)."""
    bad = []
    for l in range(case.max_level + 1):
        s = level_state(l)
        keys = np.asarray(s["keys"], np.uint64)
        if hashlib.sha256(np.ascontiguousarray(keys).tobytes()).digest() != bytes(z[f"keysha{l}"]):
            bad.append(f"level {l}: keys")
            continue
        keep = (np.asarray(s["tags"]) & TAG_BC) == 0
        fl = np.isin(keys, case.mesh.levels[l]["lat_f"])
        si = z[f"sidx{l}"]
        for what, arr, ref in (("f", s["f"][:, keep], "fsha"), ("fcol", s["fcol"], "fcolsha"),
                               ("rho", np.asarray(s["rho"])[fl], "rhosha"), ("u", np.asarray(s["u"])[:, fl], "usha")):
            if sha(arr) != bytes(z[f"{ref}_{d}_{l}"]):
                msg = f"dump {d} level {l}: {what}"
                if what in ("f", "fcol"):
                    full = s["f"] if what == "f" else s["fcol"]
                    msg += f" (sampled cells max |diff| {float(np.abs(full[:, si] - z[f's{what}_{d}_{l}']).max()):.3g})"
                bad.append(msg)
    return bad


def oracle_state(oc):
    def get(l):
        g = oc.get(l)
        g["u"] = np.ascontiguousarray(g["u"].T)
        return g
    return get


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
