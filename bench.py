"""Benchmark: uniform single-level roofline case of the LBM time step.

Workload: D3Q19 LBGK on a 256^3 fully periodic Morton-ordered grid,
Taylor-Green initial field (u0 = 0.02, wavenumber 2 pi / 256, rho = 1 plus
the pressure term), tau = 0.6.  A step is one time step of the whole grid;
the headline runs FP32 arithmetic on populations stored as FP16 deviations
f - w_q (76 B per cell update), the FP64 / FP32 / BF16 storages are timed
beside it.  Inputs stay resident in HBM (state 637 MB at FP16, larger than
the 126 MB L2, so no flush between steps).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank runs its own replica of the case on its own GPU
(the path has no exchange step; weak scaling, no collective on the data
path); the time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_EDGE = 256
Q = 19
TAU = 0.6
NU = (TAU - 0.5) / 3.0
U0 = 0.02
CONFIG_STEPS = 500  # the uniform configuration's run length
BYTES_PER_CELL = {"f64": 2 * Q * 8, "f32": 2 * Q * 4, "f16": 2 * Q * 2, "bf16": 2 * Q * 2}
WORKLOAD = "uniform 256^3 periodic Taylor-Green, D3Q19 LBGK, tau=0.6, u0=0.02"


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic(key):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            return json.load(fh).get(key)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        # samples under load: clock above the idle floor
        loaded = [v for v in sm if v > 0.5 * max(sm)] if sm else []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows for j in range(4) if r[5 + j].lower() == "active"})
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons, "samples": len(rows)}


def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=300),
                                device_id=None)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(value, world):
    """Maximum of a per-rank scalar (the step time) over all ranks; the only
    collective of the benchmark, outside the timed region."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_mlups(cells_per_rank, steps, secs_per_rank, world):
    """Whole-job MLUPS of `world` independent replicas timed as the maximum
    over ranks (weak scaling: every rank steps its own case)."""
    return world * cells_per_rank * steps / max_over_ranks(secs_per_rank, world) / 1e6


def tgv_fields():
    from mortontrie_amr_b200.case import taylor_green_fields
    from mortontrie_amr_b200.lbm import morton_order_fields
    rho, u, v, w = taylor_green_fields((N_EDGE,) * 3, U0)
    return morton_order_fields(N_EDGE, rho, u, v, w)


def make_case(storage):
    from mortontrie_amr_b200.case import uniform_box_case
    return uniform_box_case(q=Q, n=(N_EDGE,) * 3, nu=NU, storage=storage, u_ref=U0)


def time_steps(ctx, dense, steps, warmup, world, torch):
    """Device time of `steps` steps on the library's stream (= torch's
    current stream), max over ranks; returns (seconds, launches)."""
    stream = torch.cuda.current_stream()
    dense.step(warmup)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    l0 = ctx.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dense.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    launches = ctx.launch_count() - l0
    secs = e0.elapsed_time(e1) / 1e3
    return max_over_ranks(secs, world), launches


def run_ours(args):
    import torch

    from mortontrie_amr_b200.lbm import Context, DenseCase
    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    # a dedicated (non-default) stream shared by torch's events and the library
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    ctx = Context(local)
    ctx.set_stream(stream.cuda_stream)
    fields = tgv_fields()
    n_cells = N_EDGE ** 3
    peak, peak_kind = measured_hbm_peak()

    # headline: FP16 shifted storage (profiling runs: --quick --quick-storage picks another)
    hs = args.quick_storage if args.quick else "f16"
    case = make_case(hs)
    dense = DenseCase(ctx, case, hs)
    dense.init_fields(*fields)
    block, tune_ms = dense.tune()  # outside the timed region; leaves the state unchanged
    sampler = ClockSampler(local)
    if rank == 0:
        sampler.start()
    secs, launches = time_steps(ctx, dense, args.steps, args.warmup, world, torch)
    clocks = sampler.stop() if rank == 0 else None
    mlups = world * n_cells * args.steps / secs / 1e6
    per_launch = secs / args.steps
    achieved = BYTES_PER_CELL[hs] * n_cells / per_launch / 1e9
    red = dense.reduce()
    dense.close()

    # storage variants, same workload
    variants = {}
    for st in (() if args.quick else ("f64", "f32", "bf16")):
        d = DenseCase(ctx, make_case(st), st)
        d.init_fields(*fields)
        vblock, _ = d.tune()
        s, _ = time_steps(ctx, d, args.steps, args.warmup, world, torch)
        bw = BYTES_PER_CELL[st] * n_cells / (s / args.steps) / 1e9
        variants[st] = {"mlups": round(world * n_cells * args.steps / s / 1e6, 1),
                        "bytes_per_cell_update": BYTES_PER_CELL[st], "achieved_gbs": round(bw, 1),
                        "frac": round(bw / peak, 4), "block": vblock}
        d.close()

    # end to end through the public API: pinned host fields -> device, the
    # steps, density + velocity back to pinned host memory
    if args.quick:
        if rank == 0:
            print(json.dumps({"quick": True, "storage": hs, "edge": N_EDGE, "mlups": round(mlups, 1), "block": block,
                              "tune_ms": tune_ms, "achieved_gbs": round(achieved, 1),
                              "launches": int(launches)}), flush=True)
        ctx.close()
        return
    host = [torch.from_numpy(f).pin_memory() for f in fields]
    out_rho = torch.empty(n_cells, dtype=torch.float64).pin_memory()
    out_u = torch.empty(3 * n_cells, dtype=torch.float64).pin_memory()
    d = DenseCase(ctx, case, "f16")
    stream = torch.cuda.current_stream()
    d.init_fields_ptr(*[h.data_ptr() for h in host])
    d.tune()
    d.step(args.warmup)
    d.macros_ptr(out_rho.data_ptr(), out_u.data_ptr())
    torch.cuda.synchronize()
    def solve(nsteps):
        """one job through the public API: pinned FP64 rho, u in -> nsteps -> rho, u out"""
        barrier(world)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        d.init_fields_ptr(*[h.data_ptr() for h in host])
        d.step(nsteps)
        d.macros_ptr(out_rho.data_ptr(), out_u.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        barrier(world)
        secs = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
        h2d = 4 * 8 * n_cells
        d2h = 4 * 8 * n_cells
        return {"value": round(world * n_cells * nsteps / secs / 1e6, 1), "unit": "MLUPS",
                "h2d_bytes_per_step": h2d // nsteps, "d2h_bytes_per_step": d2h // nsteps,
                "h2d_bytes_per_solve": h2d, "d2h_bytes_per_solve": d2h, "steps_per_solve": nsteps,
                "wall_s": round(wall, 4),
                "path": "mt_case_init_fields (pinned FP64 rho,u) -> mt_step x steps -> mt_case_get_macros (pinned)"}

    def solve_pipelined(jobs, nsteps):
        """`jobs` jobs back to back on two cases, each on its own context and
        stream: job k+1's fields go in and its steps are queued before job
        k's results are read back, so one job's copies overlap the other's
        steps (every job still moves its inputs in and its results out).
        CUDA events: start on the first stream, end after it has waited for
        the second."""
        s2 = torch.cuda.Stream(device=local)
        ctx2 = Context(local)
        ctx2.set_stream(s2.cuda_stream)
        d2 = DenseCase(ctx2, case, "f16")
        d2.init_fields_ptr(*[h.data_ptr() for h in host])
        d2.tune()
        d2.step(args.warmup)
        out2 = (torch.empty(n_cells, dtype=torch.float64).pin_memory(),
                torch.empty(3 * n_cells, dtype=torch.float64).pin_memory())
        d2.macros_ptr(out2[0].data_ptr(), out2[1].data_ptr())
        ds, outs = [d, d2], [(out_rho, out_u), out2]
        torch.cuda.synchronize()
        barrier(world)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s2.wait_stream(stream)
        ds[0].init_fields_ptr(*[h.data_ptr() for h in host])
        ds[0].step(nsteps)
        for k in range(jobs):
            if k + 1 < jobs:
                nxt = ds[(k + 1) % 2]
                nxt.init_fields_ptr(*[h.data_ptr() for h in host])
                nxt.step(nsteps)
            o = outs[k % 2]
            ds[k % 2].macros_ptr(o[0].data_ptr(), o[1].data_ptr())
        stream.wait_stream(s2)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        secs = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
        d2.close()
        ctx2.close()
        h2d = 4 * 8 * n_cells
        return {"value": round(world * n_cells * nsteps * jobs / secs / 1e6, 1), "unit": "MLUPS", "jobs": jobs,
                "steps_per_solve": nsteps, "h2d_bytes_per_step": h2d // nsteps, "d2h_bytes_per_step": h2d // nsteps,
                "path": "two contexts alternating: job k+1 in and queued before job k's results are read"}

    # the configuration's run is 500 steps: one such job, copies included;
    # a job of the timed K steps beside it; and jobs back to back, pipelined
    e2e = solve(CONFIG_STEPS)
    e2e["k_step_job"] = solve(args.steps)
    try:
        e2e["pipelined_jobs"] = solve_pipelined(4, CONFIG_STEPS)
    except Exception as exc:  # reported, not hidden
        e2e["pipelined_jobs"] = {"error": repr(exc)}
    d.close()

    amr = None
    if not args.no_amr:
        try:
            amr = amr_section(ctx, torch)
        except Exception as exc:  # reported, not hidden: the line says why the section is missing
            amr = {"error": repr(exc)}
    octree = None
    if not args.no_amr and not args.no_octree:
        try:
            octree = octree_section(ctx, torch)
        except Exception as exc:
            octree = {"error": repr(exc)}
    served = None
    if not args.no_served and world == 1:
        try:
            served = served_section(ctx, torch)
        except Exception as exc:
            served = {"error": repr(exc)}
    batched = None
    if not args.no_batched and world == 1:
        try:
            batched = batched_section(ctx, torch)
        except Exception as exc:
            batched = {"error": repr(exc)}
    moving = None
    if not args.no_moving and world == 1:
        try:
            moving = moving_section(ctx, torch)
        except Exception as exc:
            moving = {"error": repr(exc)}

    if rank == 0:
        cpu = cpu_baseline_sample() if (world == 1 and not args.no_cpu_baseline) else None
        traffic = committed_traffic("k_dense_q19_f16_256")
        line = {
            "metric": "fine-level MLUPS (uniform case), %HBM roofline",
            "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1e3 * secs / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": n_cells, "storage": "f16 deviations f - w_q",
                       "bytes_per_cell_update": BYTES_PER_CELL["f16"], "levels": 1,
                       "block": block, "tune_ms_per_launch": tune_ms,
                       "l2": "state 637 MB > 126 MB L2; no flush", "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "k_dense_pair<19, half, LBGK> (fused pull + collide)",
                         "algorithmic_bytes_per_launch": BYTES_PER_CELL["f16"] * n_cells},
            "variants": variants,
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
            "diagnostics": {"mass": red["mass"], "kinetic_energy": red["kinetic_energy"]},
            "cpu_baseline": cpu,
            "amr_cumulant_sphere": amr,
            "amr_octree_sphere": octree,
            "batched_uneven": batched,
            "served_mix": served,
            "moving_refinement": moving,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


SHIFT_NOTE = {"inlet": "feq(1, u_bc) on every level", "far_field": "feq(1, u_bc) below the finest level, w on it"}


def _shift_of_label(label):
    """storage_shift of a run label: *_inlet, *_far or none (w)."""
    if label.endswith("_inlet"):
        return "inlet"
    if label.endswith("_far"):
        return "far_field"
    return None


def amr_section(ctx, torch, steps=10, warmup=2, only=None, tune=True):
    """4-level D3Q27 cumulant sphere (192x96x96 coarse, R = 6 coarse = 48
    finest cells, Re 200, u 0.04, nested boxes 4R / 2.5R / 1.75R): coarse
    steps of the multi-level path in the reference's FP64 and with FP32 / FP16
    storage.  Fine-level MLUPS = finest stepped cells x 2^L per coarse step;
    total MLUPS sums every level's substeps.  Accuracy of the reduced storage
    is stated against the FP64 run after the same steps."""
    from mortontrie_amr_b200.case import nested_sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    t0 = time.time()
    case = nested_sphere_case()
    host_mesh_s = time.time() - t0
    m = case.mesh
    L = m.spec.max_level
    stepped = [int(m.levels[l]["lat_f"].size + m.levels[l]["overlap_C2F"].size) for l in range(L + 1)]
    per_coarse_total = sum(n << l for l, n in enumerate(stepped))
    per_coarse_fine = stepped[L] << L
    out = {"workload": "4-level D3Q27 cumulant sphere 192x96x96, R=6 (48 finest), Re=200, u=0.04",
           "stepped_cells_per_level": stepped, "coarse_steps": steps,
           "accuracy_note": "errors vs FP64 after the warm-up, one more and the timed coarse steps from the uniform "
                            "inflow state (an impulsively started sphere: a transient drag); the long-run "
                            "comparison is bench.py --amr-accuracy"}
    stream = torch.cuda.current_stream()
    res = {}
    # (label, storage, schedule): the plain form is FP64 in the reference's
    # phase order; the reduced storages run the fused schedule
    # (*_inlet: reduced storage shifted by feq(1, u_bc) instead of w on every
    # level; *_far: on the levels below the finest)
    runs = [("f64", "f64", "phases"), ("f64_fused", "f64", "fused"), ("f32", "f32", "fused"),
            ("f16", "f16", "fused"), ("bf16", "bf16", "fused"), ("f16_phases", "f16", "phases"),
            ("f16_inlet", "f16", "fused"), ("f16_far", "f16", "fused"), ("bf16_far", "bf16", "fused")]
    if only:
        runs = [r for r in runs if r[0] in only]
    for st, storage, schedule in runs:
        mgr = LBM_Manager(ctx, case, storage, schedule=schedule,
                          storage_shift=_shift_of_label(st))
        if _shift_of_label(st):
            out[st] = {"storage_shift": SHIFT_NOTE[_shift_of_label(st)]}
        mgr.fluidSimulate(warmup)
        forms = form_ms = None
        if schedule == "fused" and tune:
            # the project autotuner picks each brick level's pass form (outside the timed region)
            forms, form_ms = mgr.tune_bricks()
        mgr.fluidSimulate(1)  # every run: captures the tuned step's graph before the timing
        torch.cuda.synchronize()
        mgr.reset_force()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        mgr.fluidSimulate(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        secs = e0.elapsed_time(e1) / 1e3
        rho, u = mgr.macros(L)
        keys, tags = mgr.keys(L)
        fluid = (tags & 1) != 0
        f = mgr.force()
        res[st] = dict(secs=secs, u=u[:, fluid], rho=rho[fluid], fx=f[0] / max(f[3], 1.0))
        out[st] = {**out.get(st, {}), "storage": storage, "schedule": schedule,
                   "fine_mlups": round(per_coarse_fine * steps / secs / 1e6, 1),
                   "total_mlups": round(per_coarse_total * steps / secs / 1e6, 1),
                   "ms_per_coarse_step": round(1e3 * secs / steps, 3)}
        if forms is not None:
            out[st]["brick_forms_per_level"] = [int(v) for v in forms]
            # ms per launch of each form (rows: levels; -1: not timed)
            out[st]["brick_form_ms"] = [[round(float(t), 4) for t in row] for row in form_ms]
        mgr.close()
    ref = res.get("f64")
    for st, _, _ in runs:
        if ref is None or st == "f64":
            continue
        r = res[st]
        out[st]["velocity_l2_vs_f64"] = float(np.linalg.norm(r["u"] - ref["u"]) / np.linalg.norm(ref["u"]))
        out[st]["drag_rel_vs_f64"] = float(abs(r["fx"] - ref["fx"]) / max(abs(ref["fx"]), 1e-300))
        out[st]["mass_drift_vs_f64"] = float(abs(r["rho"].sum() - ref["rho"].sum()) / ref["rho"].sum())
        out[st]["speedup_vs_f64"] = round(res["f64"]["secs"] / r["secs"], 3)
    # case set-up: the host mesher vs classification on the device (same
    # sets); one small case first loads the classification kernels
    LBM_Manager(ctx, nested_sphere_case(coarse=(48, 24, 24), max_level=2, center=(16, 12, 12), radius=2.0,
                                        half_widths=(4.0, 2.5), mesh="device"), "f16", schedule="fused").close()
    torch.cuda.synchronize()
    t0 = time.time()
    mgr = LBM_Manager(ctx, nested_sphere_case(mesh="device"), "f16", schedule="fused")
    torch.cuda.synchronize()
    dev_s = time.time() - t0
    same = all(np.array_equal(mgr.keys(l)[0], m.all_keys(l)) for l in range(L + 1))
    mgr.close()
    out["case_setup_s"] = {"host_mesher": round(host_mesh_s, 2), "device_classification_and_build": round(dev_s, 3),
                           "same_keys": bool(same)}
    return out


def octree_section(ctx, torch, steps=10, warmup=2, band=6.0, margin=6):
    """The 4-level D3Q27 cumulant sphere of amr_section (192x96x96 coarse,
    R = 6, Re 200) refined from the body instead of nested boxes: octree
    regions (every level-2 cell within `band` of the surface on the finest
    level, `margin` cells of each level around the next), classified on the
    device.  Cells per level, setup time, FP64 (phase order) and FP16 (fused,
    tuned brick forms) ms per coarse step."""
    from mortontrie_amr_b200.case import Octree, sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    oc = Octree(band=band, margin=margin)
    case = sphere_case(q=27, collision="Cumulant", coarse=(192, 96, 96), max_level=3, center=(64, 48, 48),
                       radius=6.0, u=0.04, re=200.0, octree=oc, mesh="device")
    out = {"workload": f"4-level D3Q27 cumulant sphere 192x96x96, R=6, Re=200, octree band {band} level-2 cells, "
                       f"margin {margin}, classified on the device"}
    stream = torch.cuda.current_stream()
    for st, storage, schedule in (("f64", "f64", "phases"), ("f16", "f16", "fused")):
        torch.cuda.synchronize()
        t0 = time.time()
        mgr = LBM_Manager(ctx, case, storage, schedule=schedule)
        torch.cuda.synchronize()
        setup = time.time() - t0
        if "stored_cells_per_level" not in out:
            out["stored_cells_per_level"] = [int(mgr.keys(l)[0].size) for l in range(mgr.L + 1)]
            out["cell_updates_per_coarse_step"] = _stepped_updates(mgr)
        mgr.fluidSimulate(warmup)
        if schedule == "fused":
            mgr.tune_bricks()
        mgr.fluidSimulate(1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        mgr.fluidSimulate(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        secs = e0.elapsed_time(e1) / 1e3
        from mortontrie_amr_b200.lbm import MTError
        try:
            mgr.status()
            finite = True
        except MTError:
            finite = False
        out[st] = {"schedule": schedule, "setup_s": round(setup, 3), "ms_per_coarse_step": round(1e3 * secs / steps, 3),
                   "total_mlups": round(out["cell_updates_per_coarse_step"] * steps / secs / 1e6, 1),
                   "finite": finite}
        mgr.close()
    return out


def _stepped_updates(mgr):
    """Cell updates of one coarse step: the stepped cells (lat_f and C2F
    tags) of every level times its 2^l substeps, read from the device build."""
    total = 0
    for l in range(mgr.L + 1):
        _, tags = mgr.keys(l)
        total += int(np.count_nonzero(tags & 5)) << l
    return total


def batched_section(ctx, torch, steps=20, warmup=2, solve_steps=2000, n_cases=64, seed=4):
    """Batched uneven instances: 64 seeded cases (cavities and spheres, 4
    domain sizes, 1-3 refinement levels, Re 10-200, D3Q19 LBGK or D3Q27
    cumulant, stress-continuous interface factors).  All cases in one batch
    (FP16 storage, fused schedule, one batched brick pass per level, substep
    and model) against the same cases solved one at a time in the plain form
    (FP64, phase order) and one at a time with FP16 storage.  Cases/h assume
    `solve_steps` coarse steps per case at the measured per-step times;
    accuracy compares the batched FP16 state with plain FP64 after the same
    number of coarse steps."""
    from mortontrie_amr_b200.lbm import Batch, LBM_Manager, drag_coefficient
    from mortontrie_amr_b200.workloads import batched_uneven_cases
    specs = batched_uneven_cases(seed, n_cases)
    # meshes classified on the device when each case is created
    cases = [s.build(mesh="device") for s in specs]
    stream = torch.cuda.current_stream()
    total_steps = warmup + steps

    def timed(fn, k):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn(k)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    # batched, FP16
    t0 = time.time()
    members = [LBM_Manager(ctx, c, "f16", schedule="fused", scaling="standard", interface_time="hold")
               for c in cases]
    torch.cuda.synchronize()
    build_s = time.time() - t0
    upd = [_stepped_updates(m) for m in members]
    t0 = time.time()
    batch = Batch(ctx, members)
    batch.step(warmup)
    torch.cuda.synchronize()
    setup_b = time.time() - t0
    tb = timed(batch.step, steps) / steps
    res_b = [_case_result(m, c) for m, c in zip(members, cases)]
    batch.close()
    for m in members:
        m.close()
    # one at a time: plain FP64, and FP16 fused
    out_single = {}
    res_p = None
    for label, storage, schedule in (("plain_f64", "f64", "phases"), ("f16_one_at_a_time", "f16", "fused")):
        per = []
        res = []
        for c in cases:
            mgr = LBM_Manager(ctx, c, storage, schedule=schedule, scaling="standard", interface_time="hold")
            mgr.fluidSimulate(warmup)
            per.append(timed(mgr.fluidSimulate, steps) / steps)
            if label == "plain_f64":
                res.append(_case_result(mgr, c))
            mgr.close()
        if label == "plain_f64":
            res_p = res
        solve = solve_steps * sum(per)
        out_single[label] = {"ms_per_coarse_step_all_cases": round(1e3 * sum(per), 3),
                             "cases_per_hour": round(len(cases) * 3600.0 / solve, 1),
                             "mlups": round(sum(upd) / sum(per) / 1e6, 1)}
    solve_b = solve_steps * tb
    l2 = [float(np.linalg.norm(b["u"] - p["u"]) / max(np.linalg.norm(p["u"]), 1e-300)) for b, p in zip(res_b, res_p)]
    finite = [bool(np.isfinite(b["u"]).all() and np.isfinite(p["u"]).all()) for b, p in zip(res_b, res_p)]
    drag = [abs(b["cd"] - p["cd"]) / abs(p["cd"]) for b, p, c in zip(res_b, res_p, cases)
            if c.mesh.spec.sphere is not None and np.isfinite(p["cd"]) and abs(p["cd"]) > 1e-6]
    fin_l2 = [x for x, f in zip(l2, finite) if f]
    return {
        "workload": f"{len(cases)} seeded cases (seed {seed}): cavity/sphere, 32^3..128x64x64, 1-3 levels, "
                    "Re 10-200, D3Q19 LBGK / D3Q27 cumulant, stress-continuous interface factors, "
                    "fine interface re-exploded in both substeps",
        "cell_updates_per_coarse_step": int(sum(upd)), "device_mesh_build_s": round(build_s, 2),
        "batch_setup_s": round(setup_b, 2), "coarse_steps_timed": steps, "solve_coarse_steps": solve_steps,
        "batched_f16": {"ms_per_coarse_step_all_cases": round(1e3 * tb, 3),
                        "cases_per_hour": round(len(cases) * 3600.0 / solve_b, 1),
                        "mlups": round(sum(upd) / tb / 1e6, 1)},
        **out_single,
        "speedup_vs_plain_one_at_a_time": round(out_single["plain_f64"]["ms_per_coarse_step_all_cases"] /
                                                (1e3 * tb), 2),
        "accuracy_after_steps": total_steps,
        "finite_cases": int(sum(finite)),
        "velocity_l2_vs_plain_f64": {"median": float(np.median(fin_l2)) if fin_l2 else None,
                                     "max": float(np.max(fin_l2)) if fin_l2 else None},
        "drag_rel_vs_plain_f64": {"median": float(np.median(drag)) if drag else None,
                                  "max": float(np.max(drag)) if drag else None, "sphere_cases": len(drag)},
    }


def _case_result(mgr, case):
    from mortontrie_amr_b200.lbm import drag_coefficient
    L = case.mesh.spec.max_level
    us = []
    for l in range(L + 1):
        _, u = mgr.macros(l)
        _, tags = mgr.keys(l)
        us.append(u[:, (tags & 1) != 0])
    cd = float("nan")
    if case.mesh.spec.sphere is not None:
        cd = drag_coefficient(mgr.force(), float(case.params.u_bc[0]), 2.0 * case.mesh.spec.sphere.radius * (1 << L))
    return {"u": np.concatenate(us, axis=1), "cd": cd}


def served_case_section(ctx, torch, steps=10, warmup=2):
    """The largest request of the served mix alone: a direct-forcing sphere
    of radius 8 coarse cells (channel 128x64x64, 3 refinement levels, 51,472
    markers), oscillating, D3Q19 LBGK, FP16 storage, fused schedule, lattice
    classified on the device.  Also the profiling driver of the forcing
    kernels (few launches: one case, `warmup` + `steps` coarse steps)."""
    from mortontrie_amr_b200.case import df_sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    from mortontrie_amr_b200.serving import AMPLITUDE, PERIOD, U_INLET
    case = df_sphere_case(radius=8, max_level=3, re=150.0, oscillating=True, u=U_INLET, period=PERIOD,
                          amplitude=AMPLITUDE, mesh="device")
    stream = torch.cuda.current_stream()
    mgr = LBM_Manager(ctx, case, "f16", schedule="fused", scaling="standard")
    upd = _stepped_updates(mgr)
    band = int(np.count_nonzero(mgr.keys(3)[1] & 256))
    mgr.fluidSimulate(warmup)
    torch.cuda.synchronize()
    n0 = ctx.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    mgr.fluidSimulate(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    out = {"workload": "DF sphere R=8 (64 finest), 128x64x64 coarse, 3 refinement levels, oscillating, Re 150, FP16",
           "cell_updates_per_coarse_step": upd, "band_cells": band, "markers": int(case.mesh.markers.dv.size),
           "coarse_steps": steps, "ms_per_coarse_step": round(1e3 * secs / steps, 3),
           "mlups": round(upd * steps / secs / 1e6, 1),
           "launches_per_coarse_step": (ctx.launch_count() - n0) // steps}
    mgr.close()
    return out


def moving_section(ctx, torch, steps=250, window=32, radius=8, max_level=3, re=100.0):
    """An oscillating direct-forcing sphere (R = 8 coarse cells, 3
    refinement levels, amplitude R/2, one period = 2000 finest = 250 coarse
    steps, FP16) on the static mesh whose finest box and forcing band cover
    the whole swept path, and with the refinement moving with the sphere
    (re-meshed every `window` coarse steps on the device, state carried by
    mt_case_remap), and on a static octree made from the forcing band over
    the path.  Wall time per coarse step (re-meshing included), cells of the
    finest level and of the band, and the mean drag and lift of the runs."""
    from mortontrie_amr_b200.case import df_sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    from mortontrie_amr_b200.moving import MovingSphere
    from mortontrie_amr_b200.serving import AMPLITUDE, PERIOD, U_INLET
    kw = dict(radius=radius, max_level=max_level, re=re, u=U_INLET, amplitude=AMPLITUDE, period=PERIOD)
    d = 2.0 * radius * (1 << max_level)
    area = np.pi * d * d / 4.0

    def coeffs(f):
        n = max(f[3], 1.0)
        return [float(2.0 * f[a] / n / (U_INLET ** 2 * area)) for a in (0, 1)]

    out = {"workload": f"oscillating DF sphere R={radius}, {max_level} refinement levels, Re {re:g}, u {U_INLET:g}, "
                       f"{steps} coarse steps (one period), FP16", "window_coarse_steps": window}
    torch.cuda.synchronize()
    t = time.perf_counter()
    st = LBM_Manager(ctx, df_sphere_case(oscillating=True, mesh="device", **kw), "f16", schedule="fused",
                     scaling="standard")
    st.fluidSimulate(steps)
    torch.cuda.synchronize()
    ws = time.perf_counter() - t
    fine_s = st.size(max_level)
    band_s = int(np.count_nonzero(st.keys(max_level)[1] & 256))
    cs = coeffs(st.force())
    st.close()
    torch.cuda.synchronize()
    t = time.perf_counter()
    mv = MovingSphere(ctx, storage="f16", window=window, **kw)
    mv.step(steps)
    torch.cuda.synchronize()
    wm = time.perf_counter() - t
    fine_m = mv.mgr.size(max_level)
    band_m = int(np.count_nonzero(mv.mgr.keys(max_level)[1] & 256))
    cm = coeffs(mv.total_force())
    out["static"] = {"ms_per_coarse_step": round(1e3 * ws / steps, 3), "finest_cells": fine_s, "band_cells": band_s,
                     "cd": cs[0], "cl": cs[1]}
    out["moving"] = {"ms_per_coarse_step": round(1e3 * wm / steps, 3), "finest_cells": fine_m, "band_cells": band_m,
                     "cd": cm[0], "cl": cm[1], "windows": mv.windows, "remesh_s": round(mv.remesh_s, 2),
                     "remesh_median_s": {k: round(float(np.median([t[i] for t in mv.remesh_times])), 4)
                                         for i, k in enumerate(("build", "remap", "release"))}}
    out["speedup"] = round(ws / wm, 3)
    out["cd_rel_diff"] = float(abs(cm[0] - cs[0]) / max(abs(cs[0]), 1e-30))
    mv.close()
    # the static mesh refined from the forcing band over the path (octree;
    # the fluid inside the sphere on coarser levels) instead of boxes
    from mortontrie_amr_b200.case import Octree
    from mortontrie_amr_b200.serving import SERVE_OCTREE
    torch.cuda.synchronize()
    t = time.perf_counter()
    so = LBM_Manager(ctx, df_sphere_case(oscillating=True, mesh="device", octree=Octree(**SERVE_OCTREE), **kw), "f16",
                     schedule="fused", scaling="standard")
    so.fluidSimulate(steps)
    torch.cuda.synchronize()
    wo = time.perf_counter() - t
    co = coeffs(so.force())
    out["static_octree"] = {"ms_per_coarse_step": round(1e3 * wo / steps, 3), "finest_cells": so.size(max_level),
                            "band_cells": int(np.count_nonzero(so.keys(max_level)[1] & 256)),
                            "cells_all_levels": int(sum(so.size(l) for l in range(max_level + 1))),
                            "cd": co[0], "cl": co[1], "speedup_vs_static": round(ws / wo, 3),
                            "cd_rel_diff_vs_static": float(abs(co[0] - cs[0]) / max(abs(cs[0]), 1e-30)),
                            "cl_abs_diff_vs_static": float(abs(co[1] - cs[1]))}
    so.close()
    return out


def served_section(ctx, torch, duration=3.0, rate=20.0, seed=5, n_fp64=4, chunk=16, refine="boxes"):
    """Served mix: a seeded Poisson stream (rate 20/s for `duration` s) of
    direct-forcing sphere flows (R in [3, 8], 16R x 8R x 8R, 1-3 refinement
    levels, Re in [20, 300], D3Q19 LBGK, half oscillating with amplitude R/2
    and period 2000 finest steps), each solved for 2000 finest steps, served
    by continuous batching in FP16 under a 150 GB budget.  Cases/h and the
    p50/p99 time-to-solution come from the wall clock of the request loop and
    count finite results only (device guard of the final state, and a finite
    drag); diverged requests are reported as failed.  The one-at-a-time rate
    solves every request of the stream alone (FP16, fused schedule, back to
    back) and counts its finite results the same way, and the plain one-at-a-time rate does so in
    the plain form (FP64, phase order; set-up plus 1/8 of each request's
    steps, scaled to all); the drag error compares served results
    with FP64 solves (phase schedule) of the lowest-Re requests whose served
    result is finite.  refine: nested boxes around each sphere and its path,
    or an octree made from its forcing band ("octree")."""
    from mortontrie_amr_b200.serving import Server, TemplateCache, plain_solve_seconds, poisson_requests, solve_alone
    reqs = poisson_requests(seed=seed, rate=rate, duration=duration)
    cache = TemplateCache(workers=max(1, min(16, (os.cpu_count() or 2) - 1)), refine=refine)
    t0 = time.time()
    cache.prepare(reqs)
    prep = time.time() - t0
    # warm the kernels and the batch path on one small request (not timed)
    Server(ctx, cache, storage="f16", chunk=chunk).run(reqs[:1], realtime=False)
    stats = Server(ctx, cache, storage="f16", budget_gb=150.0, chunk=chunk).run(reqs, realtime=True)
    served = stats.summary()
    alone = [solve_alone(ctx, cache, r, storage="f16", with_status=True) for r in reqs]
    t_alone = [a[2] for a in alone]
    ok_alone = {r.rid for r, a in zip(reqs, alone) if a[3] and np.isfinite(a[0])}
    # finite results per hour of one-at-a-time solving: the same requests, the same count rule as the served loop
    alone_rate = 3600.0 * len(ok_alone) / float(np.sum(t_alone))
    # the plain form one at a time (FP64, phase order), from 1/8 of each request's steps; finite
    # results counted as in the FP16 one-at-a-time run (the plain run is too short to tell)
    # (streams longer than 60 requests: the first 60, the rate scaled by the finite share)
    plain_reqs = reqs[:60]
    t_plain = [plain_solve_seconds(ctx, cache, r) for r in plain_reqs]
    plain_rate = 3600.0 * len(plain_reqs) * (len(ok_alone) / len(reqs)) / float(np.sum(t_plain))
    res = {r.rid: r for r in stats.results}
    finite = [r for r in stats.results if r.finite and np.isfinite(r.cd)]
    ok_served = {r.rid for r in finite}
    errs = []
    for r in sorted(finite, key=lambda x: next(q.re for q in reqs if q.rid == x.rid))[:n_fp64]:
        cd64 = solve_alone(ctx, cache, next(q for q in reqs if q.rid == r.rid), storage="f64")[0]
        if np.isfinite(cd64) and abs(cd64) > 1e-6:
            errs.append(abs(res[r.rid].cd - cd64) / abs(cd64))
    from mortontrie_amr_b200.serving import U_INLET
    return {"workload": f"{len(reqs)} Poisson requests ({rate:g}/s over {duration:g} s, seed {seed}): DF sphere "
                        f"R 3-8, 1-3 levels, Re 20-300, inlet u {U_INLET:g}, half oscillating, 2000 finest steps "
                        f"each, FP16, refinement: {refine}",
            "template_build_s": round(prep, 1), "templates": len(cache.meshes), **served,
            "finite_results": len(finite),
            "finite_alone": len(ok_alone),
            "finite_differs_alone_vs_mix": len(ok_alone ^ ok_served),
            "one_at_a_time_cases_per_hour": round(alone_rate, 1),
            "one_at_a_time_wall_s": round(float(np.sum(t_alone)), 2),
            "served_vs_one_at_a_time": round(served["cases_per_hour"] / alone_rate, 2),
            "plain_f64_one_at_a_time_cases_per_hour": round(plain_rate, 1),
            "plain_f64_sample_requests": len(plain_reqs),
            "served_vs_plain_f64_one_at_a_time": round(served["cases_per_hour"] / plain_rate, 2),
            "drag_rel_vs_fp64": {"median": float(np.median(errs)) if errs else None,
                                 "max": float(np.max(errs)) if errs else None, "sample": len(errs)}}


ACCURACY_CASES = {
    "cfg3": "4-level D3Q27 cumulant sphere 192x96x96, R=6, Re=200, u=0.04",
    "cfg3_re20": "4-level D3Q27 cumulant sphere 192x96x96, R=6, Re=20, u=0.04",
    "cfg1": "2-level D3Q19 LBGK sphere 64x32x32, R=4, Re=20, u=0.05",
}


def _accuracy_case(name):
    from mortontrie_amr_b200.case import nested_sphere_case, sphere_case
    if name == "cfg1":
        return sphere_case()
    return nested_sphere_case(re=20.0 if name == "cfg3_re20" else 200.0)


def amr_accuracy(ctx, torch, steps=2500, case_name="cfg3", scaling="reference", only=None):
    """Long-run accuracy of the reduced storages (fused schedule; shifted by
    w, or by feq(1, u_bc) on every level (*_inlet) or below the finest
    (*_far)) against the FP64 phase schedule on a
    sphere case: after `steps` coarse steps, the
    drag coefficient averaged over the last tenth of the run, the velocity
    field of every level's lat_f cells (relative L2), the total mass, and
    whether every population stayed finite."""
    from mortontrie_amr_b200.lbm import LBM_Manager, MTError, drag_coefficient
    case = _accuracy_case(case_name)
    m = case.mesh
    L = m.spec.max_level
    d_fine = 2.0 * m.spec.sphere.radius * (1 << L) if m.spec.sphere else 0.0
    u_in = float(case.params.u_bc[0])
    tail = max(steps // 10, 1)
    res = {}
    runs = [("f64", "f64", "phases"), ("f32", "f32", "fused"), ("f16", "f16", "fused"), ("bf16", "bf16", "fused"),
            ("f16_inlet", "f16", "fused"), ("f16_far", "f16", "fused"), ("bf16_far", "bf16", "fused")]
    if only:
        runs = [r for r in runs if r[0] in only or r[0] == "f64"]
    for st, storage, schedule in runs:
        mgr = LBM_Manager(ctx, case, storage, schedule=schedule, scaling=scaling,
                          storage_shift=_shift_of_label(st))
        t0 = time.time()
        mgr.fluidSimulate(steps - tail)
        mgr.reset_force()
        mgr.fluidSimulate(tail)
        torch.cuda.synchronize()
        try:
            mgr.status()
            finite = True
        except MTError:
            finite = False
        u_all, mass = [], 0.0
        for l in range(L + 1):
            rho, u = mgr.macros(l)
            _, tags = mgr.keys(l)
            fl = (tags & 1) != 0
            u_all.append(u[:, fl])
            mass += float(rho[fl].sum())
        res[st] = dict(u=np.concatenate(u_all, axis=1), u_lv=u_all, mass=mass,
                       cd=drag_coefficient(mgr.force(), u_in, d_fine), wall_s=round(time.time() - t0, 2),
                       finite=finite)
        mgr.close()
    ref = res["f64"]
    out = {"case": ACCURACY_CASES[case_name], "interface_scaling": scaling, "coarse_steps": steps,
           "finest_steps": steps << L, "drag_window_coarse_steps": tail, "cd_f64": ref["cd"],
           "f64_finite": ref["finite"]}
    for st, _, _ in runs[1:]:
        r = res[st]
        out[st] = {"cd": r["cd"], "drag_rel_vs_f64": abs(r["cd"] - ref["cd"]) / abs(ref["cd"]),
                   "velocity_l2_vs_f64": float(np.linalg.norm(r["u"] - ref["u"]) / np.linalg.norm(ref["u"])),
                   "velocity_l2_per_level": [float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
                                             for a, b in zip(r["u_lv"], ref["u_lv"])],
                   "mass_drift_vs_f64": abs(r["mass"] - ref["mass"]) / ref["mass"], "wall_s": r["wall_s"],
                   "finite": r["finite"]}
    return out


REF_EDGE = 64


def _reference_sample_case():
    """Bounded CPU sample of the workload for the reference's own code: the
    same periodic Taylor-Green D3Q19 LBGK step (tau 0.6, u0 0.02, wavenumber
    2 pi / edge) on a 64^3 box instead of 256^3 (the reference's hash maps
    hold about 2 KB per cell); the reference needs a second, empty level, and
    its periodic wrap is the harness's find_neighbor wrap."""
    from mortontrie_amr_b200.case import equilibrium, taylor_green_fields, uniform_box_case
    from mortontrie_amr_b200.lbm import morton_order_fields
    n = REF_EDGE
    case = uniform_box_case(q=Q, n=(n, n, n), nu=NU, boundary=("periodic",) * 3, empty_levels=1, u_ref=U0)
    fields = morton_order_fields(n, *taylor_green_fields((n, n, n), U0))
    f0 = equilibrium(Q, *fields)
    keys0 = case.mesh.all_keys(0)
    init = [(keys0, f0), (case.mesh.all_keys(1), np.zeros((Q, 0)))]
    return case, init


def cpu_reference_run(nprocs, steps, warmup):
    """Run `nprocs` single-threaded reference harness processes at once (one
    per core, the reference has no threading); returns (MLUPS of all
    processes, kind, cores, sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    case, init = _reference_sample_case()
    n_fluid = int(case.mesh.levels[0]["lat_f"].size)
    try:
        import oracle as O
        import build as B
        have_ref = os.path.exists(B.harness_path(Q, 1, True)) or os.path.isdir(B.REF)
    except Exception:
        have_ref = False
    if have_ref:
        with tempfile.TemporaryDirectory() as td:
            procs = [O.start_harness(case, steps, td, i, nwarm=warmup, init=init) for i in range(nprocs)]
            secs = []
            for p, out in procs:
                p.wait(timeout=3600)
                if p.returncode != 0:
                    raise RuntimeError("reference harness failed")
                with open(out, "rb") as fh:
                    secs.append(O.parse_harness_output(fh.read(), Q, 1, steps)["seconds"])
        mlups = nprocs * n_fluid * steps / max(secs) / 1e6
        kind = "reference"
    else:
        import oracle as O
        oc = O.OracleCase(case)
        oc.set_populations(0, init[0][1])
        oc.step(warmup)
        t = time.perf_counter()
        oc.step(steps)
        mlups = n_fluid * steps / (time.perf_counter() - t) / 1e6
        kind, nprocs = "port", 1
    sample = (f"{nprocs} process(es) x {steps} timed steps of a {REF_EDGE}^3 periodic Taylor-Green D3Q19 LBGK box "
              f"({n_fluid} cells each, tau 0.6), hash-map backend, 1 thread per process")
    return mlups, kind, nprocs, sample


def _case_updates(case):
    """Cell updates of one coarse step of a host-meshed case: every level's
    collide set (lat_f and overlap_F2C) times its 2^l substeps."""
    m = case.mesh
    return sum((m.levels[l]["lat_f"].size + m.levels[l]["overlap_F2C"].size) << l
               for l in range(m.spec.max_level + 1))


def cpu_reference_extras():
    """The reference's own multi-level step on the host cores for the
    multi-level configurations, one single-threaded harness process per case,
    side by side: the cfg1 geometry (64x32x32 coarse, 2 levels, sphere R 4,
    Re 20, periodic lateral sides, non-equilibrium West / East) for 3 coarse
    steps, and the 4-level D3Q27 cumulant sphere scaled by 1/4 (48x24x24
    coarse, R 1.5, Re 200, every face closed: the reference's live
    boundary) for 1 coarse step.  Each reports its seconds per coarse step,
    the 1000-step cfg1 run extrapolated from it, and MLUPS over all levels."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import oracle as O
        import build as B
    except Exception as e:  # noqa: BLE001
        return {"unavailable": f"oracle harness not importable: {e}"}
    from mortontrie_amr_b200.case import nested_sphere_case, sphere_case
    runs = {
        "cfg1_periodic": (sphere_case(bc_mode="neq"), 3),
        "cfg3_scaled_quarter": (nested_sphere_case(coarse=(48, 24, 24), center=(16, 12, 12), radius=1.5,
                                                   bc_mode="neq", boundary=("bc", "bc", "bc")), 1),
    }
    for case, _ in runs.values():
        per = any(b == "periodic" for b in case.mesh.spec.boundary)
        if not (os.path.exists(B.harness_path(case.params.q, case.mesh.spec.max_level, per)) or os.path.isdir(B.REF)):
            return {"unavailable": "the reference harness is not built"}
    out = {}
    with tempfile.TemporaryDirectory() as td:
        procs = {name: (O.start_harness(case, steps, td, name), case, steps) for name, (case, steps) in runs.items()}
        for name, ((p, path), case, steps) in procs.items():
            p.wait(timeout=1800)
            if p.returncode != 0:
                out[name] = {"unavailable": f"harness exit {p.returncode}"}
                continue
            with open(path, "rb") as fh:
                secs = O.parse_harness_output(fh.read(), case.params.q, case.mesh.spec.max_level, steps)["seconds"]
            upd = _case_updates(case)
            out[name] = {"coarse_steps": steps, "seconds_per_coarse_step": round(secs / steps, 4),
                         "total_mlups": round(upd * steps / secs / 1e6, 4), "cell_updates_per_coarse_step": upd,
                         "cores": 1}
    if "seconds_per_coarse_step" in out.get("cfg1_periodic", {}):
        out["cfg1_periodic"]["run_1000_coarse_steps_s_extrapolated"] = round(
            1000 * out["cfg1_periodic"]["seconds_per_coarse_step"], 1)
    return out


def cpu_baseline_sample():
    mlups, kind, cores, sample = cpu_reference_run(1, 10, 1)
    return {"value": round(mlups, 4), "unit": "MLUPS", "cores": cores, "kind": kind, "sample": sample,
            "per_core": round(mlups / cores, 4), "extras": cpu_reference_extras()}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    nprocs = max(1, min(os.cpu_count() or 1, 32))
    # each process times at least 10 steps (at most 20) of its box
    mlups, kind, cores, sample = cpu_reference_run(nprocs, max(10, min(args.steps, 20)), max(0, min(args.warmup, 2)))
    line = {
        "impl": "reference", "metric": "fine-level MLUPS (uniform case), %HBM roofline", "value": round(mlups, 4),
        "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": sample},
        "cpu_baseline": {"value": round(mlups, 4), "unit": "MLUPS", "cores": cores, "kind": kind, "sample": sample,
                         "per_core": round(mlups / cores, 4)},
        "e2e": {"value": round(mlups, 4), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-amr", action="store_true", help="skip the 4-level cumulant sphere section")
    ap.add_argument("--amr-only", action="store_true",
                    help="only the 4-level cumulant sphere section (K coarse steps per storage; profiling runs)")
    ap.add_argument("--no-octree", action="store_true", help="skip the octree-refined sphere section")
    ap.add_argument("--served-refine", default="boxes", choices=["boxes", "octree"],
                    help="refinement of the served requests (--served-only runs)")
    ap.add_argument("--octree-only", action="store_true", help="only the octree-refined sphere section")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched uneven instances section")
    ap.add_argument("--no-served", action="store_true", help="skip the served mix section")
    ap.add_argument("--served-only", type=float, default=0.0, metavar="SECONDS",
                    help="only the served mix, with SECONDS of Poisson arrivals")
    ap.add_argument("--batched-only", action="store_true", help="only the batched uneven instances section")
    ap.add_argument("--no-moving", action="store_true", help="skip the moving-refinement section")
    ap.add_argument("--moving-only", action="store_true", help="only the moving-refinement section")
    ap.add_argument("--served-case", action="store_true",
                    help="only the largest served request alone (profiling driver of the forcing kernels)")
    ap.add_argument("--amr-variants", default=None,
                    help="comma list of multi-level runs to time (default all: "
                         "f64,f64_fused,f32,f16,bf16,f16_phases,f16_inlet,f16_far,bf16_far); profiling and "
                         "accuracy runs")
    ap.add_argument("--amr-accuracy", type=int, default=0, metavar="N",
                    help="only the long-run accuracy of the reduced storages on the 4-level sphere (N coarse steps)")
    ap.add_argument("--accuracy-case", default="cfg3", choices=sorted(ACCURACY_CASES))
    ap.add_argument("--scaling", default="reference", choices=["reference", "standard"],
                    help="interface rescaling of the accuracy run")
    ap.add_argument("--edge", type=int, default=256, help="cube edge (power of two); 256 is the configuration")
    ap.add_argument("--quick", action="store_true", help="headline kernel only (profiling runs)")
    ap.add_argument("--quick-storage", default="f16", choices=sorted(BYTES_PER_CELL),
                    help="storage of the --quick run's kernel")
    ap.add_argument("--no-brick-tune", action="store_true",
                    help="4-level section: keep each storage's default brick form (launch-list captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    global N_EDGE
    N_EDGE = args.edge
    if args.impl == "reference":
        run_reference(args)
    elif args.served_only:
        import torch

        from mortontrie_amr_b200.lbm import Context
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx = Context(0)
        ctx.set_stream(stream.cuda_stream)
        print(json.dumps({"served_mix": served_section(ctx, torch, duration=args.served_only,
                                                       refine=args.served_refine)}), flush=True)
        ctx.close()
    elif args.moving_only:
        import torch

        from mortontrie_amr_b200.lbm import Context
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx = Context(0)
        ctx.set_stream(stream.cuda_stream)
        print(json.dumps({"moving_refinement": moving_section(ctx, torch)}), flush=True)
        ctx.close()
    elif args.served_case:
        import torch

        from mortontrie_amr_b200.lbm import Context
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx = Context(0)
        ctx.set_stream(stream.cuda_stream)
        print(json.dumps({"served_case": served_case_section(ctx, torch, steps=args.steps, warmup=2)}), flush=True)
        ctx.close()
    elif args.batched_only:
        import torch

        from mortontrie_amr_b200.lbm import Context
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx = Context(0)
        ctx.set_stream(stream.cuda_stream)
        print(json.dumps({"batched_uneven": batched_section(ctx, torch, steps=args.steps)}), flush=True)
        ctx.close()
    elif args.amr_accuracy:
        import torch

        from mortontrie_amr_b200.lbm import Context
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx = Context(0)
        ctx.set_stream(stream.cuda_stream)
        only = set(args.amr_variants.split(",")) if args.amr_variants else None
        print(json.dumps({"amr_accuracy": amr_accuracy(ctx, torch, args.amr_accuracy, args.accuracy_case,
                                                       args.scaling, only)}), flush=True)
        ctx.close()
    elif args.amr_only:
        import torch

        from mortontrie_amr_b200.lbm import Context
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx = Context(0)
        ctx.set_stream(stream.cuda_stream)
        only = args.amr_variants.split(",") if args.amr_variants else None
        print(json.dumps({"amr_cumulant_sphere": amr_section(ctx, torch, steps=args.steps, warmup=1, only=only,
                                                                       tune=not args.no_brick_tune)}),
              flush=True)
        ctx.close()
    elif args.octree_only:
        import torch

        from mortontrie_amr_b200.lbm import Context
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx = Context(0)
        ctx.set_stream(stream.cuda_stream)
        print(json.dumps({"amr_octree_sphere": octree_section(ctx, torch, steps=min(args.steps, 20))}), flush=True)
        ctx.close()
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
