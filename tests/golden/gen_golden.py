"""Generate the golden vectors under tests/golden/ by running the reference's
own LBM translation units (oracle/refharness, built by oracle/build.py from
the reference checkout) on seeded synthetic cases.

Run here, where the reference checkout exists:
    python tests/golden/gen_golden.py            # short cases + Morton answers
    python tests/golden/gen_golden.py --trace [name ...]   # TRACE_CASES
    python tests/golden/gen_golden.py --morton             # neighbour blocks
    python tests/golden/gen_golden.py --tecplot            # the reference's flow file
    python tests/golden/gen_golden.py --dis                # STL link wall distances
    python tests/golden/gen_golden.py --collide            # single-cell collision answers
    python tests/golden/gen_golden.py --tgv                # periodic Taylor-Green box
The outputs are small .npz files; the GPU box only reads them.  The trace
cases run one harness process each, in parallel; cfg1's 1000 coarse steps
take about half an hour of one core.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from mortontrie_amr_b200.case import perturbed_populations  # noqa: E402
from golden_cases import GOLDEN_CASES, TRACE_CASES, build_case  # noqa: E402


def set_digest(case):
    h = hashlib.sha256()
    m = case.mesh
    for l in range(m.spec.max_level + 1):
        for name in sorted(m.levels[l]):
            h.update(name.encode())
            h.update(np.ascontiguousarray(m.levels[l][name], np.uint64).tobytes())
    for b in m.lat_bc:
        h.update(np.ascontiguousarray(b, np.uint64).tobytes())
    h.update(np.ascontiguousarray(m.dis_keys, np.uint64).tobytes())
    h.update(np.ascontiguousarray(m.dis_rows, np.float64).tobytes())
    return h.hexdigest()


def main():
    import oracle as O
    for name, spec in GOLDEN_CASES.items():
        case = build_case(spec)
        init = perturbed_populations(case, seed=spec["seed"]) if spec["init"] == "perturbed" else None
        out = O.run_harness(case, spec["steps"], init)
        arrays = {"tau": out["tau"], "force": out["force"]}
        for l, lv in enumerate(out["levels"]):
            arrays[f"keys{l}"] = lv["keys"]
            arrays[f"f{l}"] = lv["f"]
            # fcol is compared bit-for-bit, so its SHA-256 is as strict as the array
            arrays[f"fcol_sha{l}"] = np.frombuffer(hashlib.sha256(np.ascontiguousarray(lv["fcol"]).tobytes()).digest(),
                                                   np.uint8)
        meta = dict(spec=spec, set_digest=set_digest(case))
        arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **arrays)
        print(name, os.path.getsize(path), "bytes", [lv["keys"].size for lv in out["levels"]])

    # Morton neighbour-key known answers from Morton_Assist::find_neighbor
    rng = np.random.default_rng(99)
    from mortontrie_amr_b200.lattice import cell_key
    for (q, L) in [(27, 2)]:
        levels, keys = [], []
        for l in range(L + 1):
            n = 64 << l
            x = rng.integers(0, n, 120)
            y = rng.integers(0, n, 120)
            z = rng.integers(0, n, 120)
            # include the box corners, where the masked arithmetic wraps
            x[:4], y[:4], z[:4] = [0, n - 1, 0, n - 1], [0, 0, n - 1, n - 1], [0, n - 1, n - 1, 0]
            keys.append(cell_key(L, l, x, y, z))
            levels.append(np.full(120, l, np.int32))
        levels = np.concatenate(levels)
        keys = np.concatenate(keys)
        nb = O.run_harness_morton(q, L, levels, keys)
        path = os.path.join(HERE, f"morton_kat_q{q}_l{L}.npz")
        np.savez_compressed(path, levels=levels, keys=keys, neighbors=nb)
        print("morton kat", os.path.getsize(path), "bytes")


def morton_blocks():
    """Known answers of Morton_Assist::find_neighbor for every cell of two
    8^3 blocks per level -- at the origin (every -1 step underflows a
    coordinate field) and straddling 32 * 2^l on every axis (the +1 / -1
    steps carry across five bits) -- for D3Q19 with 2 levels and D3Q19 /
    D3Q27 with 4 levels."""
    import oracle as O
    from mortontrie_amr_b200.lattice import cell_key
    for (q, L) in [(19, 1), (19, 3), (27, 3)]:
        levels, keys = [], []
        for l in range(L + 1):
            for lo in (0, (32 << l) - 4):
                r = np.arange(lo, lo + 8)
                X, Y, Z = np.meshgrid(r, r, r, indexing="ij")
                keys.append(cell_key(L, l, X.ravel(), Y.ravel(), Z.ravel()))
                levels.append(np.full(X.size, l, np.int32))
        levels = np.concatenate(levels)
        keys = np.concatenate(keys)
        nb = O.run_harness_morton(q, L, levels, keys)
        path = os.path.join(HERE, f"morton_blocks_q{q}_l{L}.npz")
        np.savez_compressed(path, levels=levels, keys=keys, neighbors=nb)
        print("morton blocks", q, L, keys.size, os.path.getsize(path), "bytes")


def tecplot_golden():
    """The reference's own flow file (IO_TECPLOTH::write, tecplot.cpp:16-176)
    after 3 coarse steps of the sphere_q19_fh_refinit case, written at
    iteration 7."""
    import oracle as O
    spec = GOLDEN_CASES["sphere_q19_fh_refinit"]
    case = build_case(spec)
    name, text = O.run_harness_tecplot(case, 3, 7)
    meta = dict(case="sphere_q19_fh_refinit", steps=3, iteration=7, file=name, set_digest=set_digest(case))
    path = os.path.join(HERE, "tecplot_sphere_q19_fh_refinit.npz")
    np.savez_compressed(path, text=np.frombuffer(text.encode(), np.uint8),
                        meta=np.frombuffer(json.dumps(meta).encode(), np.uint8))
    print("tecplot", name, os.path.getsize(path), "bytes")


DIS_CASES = {
    # off-centre icospheres: links cross faces, edges and vertices at generic angles
    "dis_icosphere_q19": dict(q=19, center=(12.3, 8.1, 7.9), radius=2.2, sub=3),
    "dis_icosphere_q27": dict(q=27, center=(12.3, 8.1, 7.9), radius=2.2, sub=3),
}


def dis_cells(spec, mesh):
    """The finest fluid cells within 1.2 coarse cells of the sphere's surface:
    every cell with a link across it and a shell of cells without one."""
    from mortontrie_amr_b200.lattice import cell_coords
    L = mesh.spec.max_level
    keys = mesh.levels[L]["lat_f"]
    x, y, z = cell_coords(L, L, keys)
    c = (np.stack([x, y, z], 1) + 0.5) / 2 ** L
    r = np.linalg.norm(c - np.asarray(spec["center"]), axis=1)
    sel = np.abs(r - spec["radius"]) < 1.2
    return keys[sel], c[sel]


def dis_golden():
    """Per link wall distances of the cells near an STL sphere by the
    reference's own Lat_Manager::compute_distance (Lat_Voxelize.cpp
    :1252-1285) over every triangle, in coarse units as the reference stores
    the surface."""
    import oracle as O
    from golden_cases import dis_mesh
    for name, spec in DIS_CASES.items():
        mesh, tris = dis_mesh(spec)
        keys, centers = dis_cells(spec, mesh)
        ref = O.run_harness_dis(spec["q"], mesh.spec.max_level, tris, keys, centers)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, keys=keys, dis=ref,
                            meta=np.frombuffer(json.dumps(spec).encode(), np.uint8))
        print("dis", name, keys.size, int((ref != -1).sum()), os.path.getsize(path), "bytes")


def collide_golden():
    """Single-cell collision known answers from the reference's own
    Collision_LBGK / Collision_Cumulant (one coarse step of a closed box):
    the sampled interior cells' populations before and after collision."""
    import oracle as O
    from golden_cases import COLLIDE_CASES, COLLIDE_SEED, collide_case, collide_sample, collide_state
    for name, spec in COLLIDE_CASES.items():
        case = collide_case(spec)
        init = collide_state(case)
        out = O.run_harness(case, 1, init)
        keys = case.mesh.all_keys(0)
        assert np.array_equal(out["levels"][0]["keys"], keys)
        idx = collide_sample(case)
        meta = dict(spec=spec, seed=COLLIDE_SEED)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, keys=keys[idx], f_in=init[0][1][:, idx], fcol=out["levels"][0]["fcol"][:, idx],
                            meta=np.frombuffer(json.dumps(meta).encode(), np.uint8))
        print("collide", name, os.path.getsize(path), "bytes")


def tgv_golden():
    """The uniform periodic Taylor-Green configuration (Morton order; D3Q19
    LBGK at 32^3 and D3Q27 cumulant at 16^3, tau 0.6, u0 0.02) after 10
    steps of the reference's own code (the periodic harness, an empty second
    level): SHA-256 of f and fcol over every cell and 64 sampled cells in
    full."""
    import tempfile
    import oracle as O
    from golden_cases import TGV_CASES, tgv_reference_case
    for name, spec in TGV_CASES.items():
        case, init = tgv_reference_case(spec)
        with tempfile.TemporaryDirectory() as td:
            p, path = O.start_harness(case, spec["steps"], td, 0, init=init)
            p.wait(timeout=3600)
            assert p.returncode == 0
            with open(path, "rb") as fh:
                out = O.parse_harness_output(fh.read(), spec["q"], 1, spec["steps"])
        lv = out["levels"][0]
        assert np.array_equal(lv["keys"], init[0][0])
        rng = np.random.default_rng(7)
        idx = np.sort(rng.choice(lv["keys"].size, size=64, replace=False))
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, fsha=_sha(lv["f"]), fcolsha=_sha(lv["fcol"]), idx=idx, f=lv["f"][:, idx],
                            fcol=lv["fcol"][:, idx], meta=np.frombuffer(json.dumps(spec).encode(), np.uint8))
        print("tgv", name, os.path.getsize(path), "bytes", round(out["seconds"], 1), "s")


SAMPLE = 64


def trace_arrays(case, out, seed=1):
    """What a trace golden keeps: per dump and level the SHA-256 of f on the
    non-boundary cells (boundary-cell f depends on the reference's hash-set
    order, and no fluid cell reads it), of fcol, of rho and u on the lat_f
    cells, and SAMPLE cells in full; the per-step force series; tau."""
    m = case.mesh
    L = m.spec.max_level
    arrays = {"tau": out["tau"], "force": out["force"]}
    bc = np.sort(np.concatenate([np.asarray(b, np.uint64) for b in m.lat_bc]))
    rng = np.random.default_rng(seed)
    for l in range(L + 1):
        keys = out["states"][0][l]["keys"]
        arrays[f"keysha{l}"] = _sha(keys.astype(np.uint64))
        n = keys.size
        arrays[f"sidx{l}"] = np.sort(rng.choice(n, size=min(SAMPLE, n), replace=False)).astype(np.int64)
    for d, st in enumerate(out["states"]):
        for l in range(L + 1):
            lv = st[l]
            keys = lv["keys"]
            keep = ~np.isin(keys, bc) if l == 0 else np.ones(keys.size, bool)
            fl = np.isin(keys, m.levels[l]["lat_f"])
            arrays[f"fsha_{d}_{l}"] = _sha(lv["f"][:, keep])
            arrays[f"fcolsha_{d}_{l}"] = _sha(lv["fcol"])
            arrays[f"rhosha_{d}_{l}"] = _sha(lv["rho"][fl])
            arrays[f"usha_{d}_{l}"] = _sha(lv["u"][:, fl])
            si = arrays[f"sidx{l}"]
            arrays[f"sf_{d}_{l}"] = lv["f"][:, si]
            arrays[f"sfcol_{d}_{l}"] = lv["fcol"][:, si]
            arrays[f"finite_{d}_{l}"] = np.array([np.isfinite(lv["f"]).all()])
    return arrays


def _sha(a):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


def gen_trace(name):
    import oracle as O
    spec = TRACE_CASES[name]
    case = build_case(spec)
    init = perturbed_populations(case, seed=spec["seed"]) if spec["init"] == "perturbed" else None
    out = O.run_harness_trace(case, spec["dumps"], init, timeout=4 * 3600)
    arrays = trace_arrays(case, out)
    meta = dict(spec=spec, set_digest=set_digest(case), seconds=out["seconds"])
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **arrays)
    return name, os.path.getsize(path), out["seconds"]


if __name__ == "__main__":
    if "--morton" in sys.argv:
        morton_blocks()
    elif "--tecplot" in sys.argv:
        tecplot_golden()
    elif "--dis" in sys.argv:
        dis_golden()
    elif "--collide" in sys.argv:
        collide_golden()
    elif "--tgv" in sys.argv:
        tgv_golden()
    elif "--trace" in sys.argv:
        from concurrent.futures import ProcessPoolExecutor
        import multiprocessing as mp
        names = [a for a in sys.argv[1:] if not a.startswith("--")] or sorted(TRACE_CASES)
        with ProcessPoolExecutor(max_workers=len(names), mp_context=mp.get_context("spawn")) as ex:
            for r in ex.map(gen_trace, names):
                print(*r, flush=True)
    else:
        main()
