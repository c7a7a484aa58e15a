"""Request loop for served sphere-flow cases (continuous batching).

Each request is a flow past a direct-forcing sphere (Lagrangian markers,
3-point kernel): radius R coarse cells, coarse channel 16R x 8R x 8R, 1 to 3
refinement levels, Reynolds number Re, D3Q19 LBGK, optionally oscillating
transversely with amplitude R/2 and a period of 2000 finest steps.  A
request is solved when its case has advanced `finest_steps` finest-level
steps (one oscillation period by default); its result is the mean drag and
lift coefficients over the run.

The server keeps every admitted case resident on the device and steps all
of them together in one batch (mt_batch_*): a request that arrives while
others are running is admitted as soon as the HBM budget allows and joins
the batch at the next chunk boundary; a finished case leaves it and frees
its memory.  Meshes come from templates keyed by the grid radius ceil(R),
the level count and whether the sphere oscillates (domain and refinement
boxes).  By default the lattice is classified on the device per request
(mt_case_generate, tens of milliseconds), with the forcing band fitted to the
request's exact radius and amplitude; with host meshes the template's band
covers any radius in [ceil(R) - 1, ceil(R)] and the cache keeps the sets.
The markers are made per request for its exact radius.
"""
from __future__ import annotations

import dataclasses
import math
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .case import CaseParams, df_sphere_case
from .mesh import Markers, SpecMesh, Sphere, estimate_cells

PERIOD = 2000          # finest steps of one oscillation
AMPLITUDE = 0.5        # oscillation amplitude in sphere radii
# inlet velocity, lattice units (every level): nu = U 2R / Re puts the
# coarse relaxation time at 0.5 + 6 U R / Re, and with LBGK and the
# reference's interface transfers the requests closest to tau = 1/2 grow
# unstable; 0.1 (Mach 0.17) doubles the finite share of the seeded stream
# over 0.05
U_INLET = 0.1
# the fine interface cells of every request are re-exploded in the second
# substep too (MT_ITIME_HOLD): with the reference's first-substep-only
# explosion 18 of the 60 requests of the seeded 20/s stream stay finite, with
# this 59 (FP16, solved alone)
INTERFACE_TIME = "hold"


@dataclass
class Request:
    rid: int
    arrival: float         # seconds after the start of the stream
    radius: float          # coarse cells
    levels: int            # refinement levels (max_level)
    re: float
    oscillating: bool
    finest_steps: int = PERIOD

    @property
    def grid_radius(self) -> int:
        return int(math.ceil(self.radius))

    def coarse_steps(self) -> int:
        return max(1, self.finest_steps >> self.levels)


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    cd: float
    cl: float
    coarse_steps: int
    storage: str
    finite: bool = True    # the device guard found no NaN / Inf population when it finished

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def poisson_requests(seed: int = 5, rate: float = 20.0, duration: float = 300.0, radius=(3.0, 8.0),
                     levels=(1, 3), re=(20.0, 300.0), p_osc: float = 0.5,
                     finest_steps: int = PERIOD) -> list:
    """Seeded Poisson stream: exponential inter-arrival times of mean 1/rate
    over `duration` seconds; R, Re uniform, levels uniform in [levels[0],
    levels[1]], oscillating with probability p_osc."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > duration:
            break
        out.append(Request(rid=len(out), arrival=t, radius=float(rng.uniform(*radius)),
                           levels=int(rng.integers(levels[0], levels[1] + 1)), re=float(rng.uniform(*re)),
                           oscillating=bool(rng.random() < p_osc), finest_steps=finest_steps))
    return out


def template_key(req: Request) -> tuple:
    return (req.grid_radius, req.levels, req.oscillating)


# refinement of a request when made from its body: the finest level covers
# the forcing band over the path and 2 level-(L-1) cells around it, each
# coarser level the next with 4 cells of margin
SERVE_OCTREE = dict(band=2.0, margin=4)


def build_template(key: tuple, mesh: str = "host", refine: str = "boxes"):
    """Mesh of a template: the host mesher's sets ("host", picklable for
    worker processes) or the spec alone ("device"); refinement in nested
    boxes around the sphere and its path, or an octree made from its forcing
    band ("octree")."""
    from .mesh import Octree
    r, levels, osc = key
    if refine not in ("boxes", "octree"):
        raise ValueError(f"refine must be 'boxes' or 'octree', not {refine!r}")
    return df_sphere_case(radius=r, max_level=levels, re=100.0, oscillating=osc, period=PERIOD,
                          amplitude=AMPLITUDE, band_slack=1.0, mesh=mesh,
                          octree=Octree(**SERVE_OCTREE) if refine == "octree" else None).mesh


def _build_host_template(key_refine: tuple):
    key, refine = key_refine
    return build_template(key, "host", refine)


def request_case(req: Request, mesh):
    """The case of one request on a template mesh: its own viscosity and
    markers (exact radius and oscillation amplitude)."""
    from .case import Case
    s = 1 << req.levels
    r = req.radius * s
    nm = max(1, int(round(4.0 * np.pi * r * r)))
    i = np.arange(nm) + 0.5
    zc = 1.0 - 2.0 * i / nm
    rc = np.sqrt(np.maximum(0.0, 1.0 - zc * zc))
    phi = i * (np.pi * (3.0 - np.sqrt(5.0)))
    ref = np.ascontiguousarray(np.stack([r * rc * np.cos(phi), r * rc * np.sin(phi), r * zc]))
    dv = np.full(nm, 4.0 * np.pi * r * r / nm)
    if req.oscillating:
        amp = AMPLITUDE * r
        t = np.arange(PERIOD)
        path = np.zeros((PERIOD, 6))
        path[:, 1] = amp * np.sin(2.0 * np.pi * t / PERIOD)
        path[:, 4] = amp * (2.0 * np.pi / PERIOD) * np.cos(2.0 * np.pi * t / PERIOD)
    else:
        path = np.zeros((1, 6))
    center = tuple(float(c * s) for c in mesh.spec.sphere.center)
    mk = Markers(ref=ref, dv=dv, center=center, path=np.ascontiguousarray(path))
    u = U_INLET
    params = CaseParams(q=19, collision="LBGK", ib_method="DF", bc_mode="zouhe_outflow",
                        nu=u * 2.0 * req.radius / req.re, u_bc=(u, 0.0, 0.0), u_ref=u)
    if isinstance(mesh, SpecMesh):
        # the band of this request's own sphere and path
        spec = dataclasses.replace(mesh.spec, sphere=Sphere(mesh.spec.sphere.center, req.radius), band_slack=0.0,
                                   oscillation=(AMPLITUDE * req.radius, PERIOD) if req.oscillating else None)
        return Case(SpecMesh(spec=spec, markers=mk), params)
    return Case(dataclasses.replace(mesh, markers=mk), params)


def footprint_bytes(case, storage: str) -> int:
    """Device memory of a resident case: three population buffers, the
    neighbour table, macros, tags and lists, bricks and halo tables."""
    sb = {"f64": 8, "f32": 4, "f16": 2, "bf16": 2}[storage]
    q = case.params.q
    total = 0
    if isinstance(case.mesh, SpecMesh):
        cells = estimate_cells(case.mesh.spec)
    else:
        cells = [sum(int(v.size) for v in lv.values()) for lv in case.mesh.levels]
    for n in cells:
        total += n * (3 * q * sb + 4 * (q - 1) + 4 * 4 + 8 + 4 + 16 + 8 + 20)
    total += int(case.mesh.markers.dv.size) * 80 if case.mesh.markers is not None else 0
    return total + (8 << 20)


def drag_lift(mgr, req: Request) -> tuple:
    return drag_lift_of(mgr.force(), req)


def drag_lift_of(f, req: Request) -> tuple:
    """Mean drag and lift coefficients from an accumulated force (fx, fy, fz, count)."""
    n = max(f[3], 1.0)
    u = U_INLET
    d = 2.0 * req.radius * (1 << req.levels)
    area = np.pi * d * d / 4.0
    return 2.0 * f[0] / n / (u * u * area), 2.0 * f[1] / n / (u * u * area)


class TemplateCache:
    """Templates by key; mesh "device" keeps specs only (the lattice is
    classified on the device per request), "host" the host mesher's sets."""

    def __init__(self, workers: int = 0, mesh: str = "device", refine: str = "boxes"):
        self.meshes = {}
        self.workers = workers
        self.mesh = mesh
        self.refine = refine

    def prepare(self, requests):
        """Build every template the requests need (host sets in worker processes)."""
        keys = sorted({template_key(r) for r in requests} - set(self.meshes))
        if not keys:
            return
        if self.mesh == "host" and self.workers > 1 and len(keys) > 1:
            import multiprocessing as mp
            from concurrent.futures import ProcessPoolExecutor
            with ProcessPoolExecutor(max_workers=min(self.workers, len(keys)),
                                     mp_context=mp.get_context("spawn")) as ex:
                for k, m in zip(keys, ex.map(_build_host_template, [(k, self.refine) for k in keys])):
                    self.meshes[k] = m
        else:
            for k in keys:
                self.meshes[k] = build_template(k, self.mesh, self.refine)

    def get(self, req: Request):
        k = template_key(req)
        if k not in self.meshes:
            self.meshes[k] = build_template(k, self.mesh, self.refine)
        return self.meshes[k]


@dataclass
class ServerStats:
    results: list = field(default_factory=list)
    wall_s: float = 0.0
    max_resident: int = 0
    max_bytes: int = 0
    chunks: int = 0
    admit_s: float = 0.0    # host time creating and building admitted cases
    step_s: float = 0.0     # host time issuing batch steps (graph capture included)
    drain_s: float = 0.0    # host time waiting for the device (queue full, no arrival) and releasing memory

    def summary(self) -> dict:
        """cases/h, p50 and p99 count the requests whose result is finite
        (the guard of their state and their drag); diverged ones are counted
        apart as failed."""
        good = [r for r in self.results if r.finite and np.isfinite(r.cd)]
        lat = np.array([r.latency for r in good]) if good else np.zeros(1)
        return {"completed": len(self.results), "finite": len(good), "failed": len(self.results) - len(good),
                "wall_s": round(self.wall_s, 2),
                "cases_per_hour": round(3600.0 * len(good) / max(self.wall_s, 1e-9), 1),
                "p50_s": round(float(np.percentile(lat, 50)), 3), "p99_s": round(float(np.percentile(lat, 99)), 3),
                "max_resident_cases": self.max_resident, "max_resident_gb": round(self.max_bytes / 1e9, 2),
                "chunks": self.chunks, "admit_s": round(self.admit_s, 2), "step_s": round(self.step_s, 2),
                "drain_s": round(self.drain_s, 2)}


class Server:
    """Continuous-batching request loop on one device context.

    The loop never synchronises the context while it runs: it keeps at most
    `max_inflight` batch chunks queued on the device (stream markers tell it
    when one has passed), admits arrivals while the device works, and learns
    that a finished request's result is ready from a marker recorded after an
    asynchronous copy of its force.  A finished case leaves the batch at once
    but keeps its memory until the budget needs it (releasing device memory
    waits for the whole device)."""

    def __init__(self, ctx, cache: TemplateCache, storage: str = "f16", budget_gb: float = 150.0,
                 chunk: int = 16, scaling: str = "standard", max_inflight: int = 2, priority_builds: bool = True,
                 storage_shift=None, interface_time: str = INTERFACE_TIME):
        self.interface_time = interface_time
        self.ctx = ctx
        self.storage_shift = storage_shift  # per-level storage shift of every case (LBM_Manager)
        self.priority_builds = priority_builds
        self.cache = cache
        self.storage = storage
        self.budget = int(budget_gb * 1e9)
        self.chunk = chunk
        self.scaling = scaling
        self.max_inflight = max_inflight

    def run(self, requests, realtime: bool = True, clock=None) -> ServerStats:
        from collections import deque

        from .lbm import Batch, Context, LBM_Manager
        stats = ServerStats()
        # admitted cases are built on a context of their own, so that the
        # build's synchronisations do not wait for the batch's queued steps
        builder = Context(self.ctx.device)
        if self.priority_builds:
            # the builds' short kernels are scheduled ahead of the batch's
            builder.set_priority(True)
        pending = sorted(requests, key=lambda r: r.arrival)
        batch = Batch(self.ctx)
        live = {}        # rid -> [mgr, req, remaining, admitted, bytes]
        finishing = []   # [marker, mgr, req, admitted, bytes]: force copy queued
        closing = []     # [mgr, bytes]: results read, memory not yet released
        inflight = deque()
        used = 0
        t0 = time.perf_counter() if clock is None else clock()
        now = (lambda: time.perf_counter() - t0) if clock is None else (lambda: clock() - t0)
        qi = 0
        while qi < len(pending) or live or finishing:
            progressed = False
            # results whose copies have landed
            for ent in list(finishing):
                if self.ctx.marker_done(ent[0]):
                    _, mgr, req, adm, need = ent
                    cd, cl = drag_lift_of(mgr.force_copied(), req)
                    stats.results.append(Result(rid=req.rid, arrival=req.arrival, admitted=adm, finished=now(),
                                                cd=cd, cl=cl, coarse_steps=req.coarse_steps(), storage=self.storage,
                                                finite=mgr.finite_copied()))
                    finishing.remove(ent)
                    closing.append([mgr, need])
                    progressed = True
            # admit arrivals as memory allows (oldest first)
            t = now() if realtime else float("inf")
            while qi < len(pending) and pending[qi].arrival <= t:
                req = pending[qi]
                case = request_case(req, self.cache.get(req))
                need = footprint_bytes(case, self.storage)
                if (live or finishing or closing) and used + need > self.budget:
                    if not closing:
                        break
                    td = time.perf_counter()
                    for mgr, nb in closing:
                        mgr.close()
                        used -= nb
                    closing = []
                    stats.drain_s += time.perf_counter() - td
                    continue
                ta = time.perf_counter()
                mgr = LBM_Manager(builder, case, self.storage, schedule="fused", scaling=self.scaling,
                                  storage_shift=self.storage_shift, interface_time=self.interface_time)
                mgr.prepare()
                mgr.transfer(self.ctx)
                batch.add(mgr)
                stats.admit_s += time.perf_counter() - ta
                live[req.rid] = [mgr, req, req.coarse_steps(), now(), need]
                used += need
                qi += 1
                progressed = True
            stats.max_resident = max(stats.max_resident, len(live))
            stats.max_bytes = max(stats.max_bytes, used)
            # issue the next chunk while the device queue has room
            while inflight and self.ctx.marker_done(inflight[0]):
                inflight.popleft()
            if live and len(inflight) < self.max_inflight:
                k = min(self.chunk, min(v[2] for v in live.values()))
                ts = time.perf_counter()
                batch.step(k)
                inflight.append(self.ctx.marker())
                stats.step_s += time.perf_counter() - ts
                stats.chunks += 1
                for v in live.values():
                    v[2] -= k
                for rid in [rid for rid, v in live.items() if v[2] == 0]:
                    mgr, req, _, adm, need = live.pop(rid)
                    mgr.force_async()
                    finishing.append([self.ctx.marker(), mgr, req, adm, need])
                    batch.remove(mgr)
                continue
            if not progressed:
                # wait for the device or the next arrival
                td = time.perf_counter()
                time.sleep(0.0005)
                stats.drain_s += time.perf_counter() - td
        self.ctx.synchronize()
        stats.wall_s = now()
        for mgr, _ in closing:
            mgr.close()
        batch.close()
        builder.close()
        return stats


def solve_alone(ctx, cache: TemplateCache, req: Request, storage: str = "f16", scaling: str = "standard",
                schedule: Optional[str] = None, storage_shift=None, with_status: bool = False,
                interface_time: str = INTERFACE_TIME) -> tuple:
    """One request by itself (no batch); returns (cd, cl, seconds), and
    whether the state stayed finite (the device guard) with with_status."""
    from .lbm import LBM_Manager, MTError
    case = request_case(req, cache.get(req))
    t = time.perf_counter()
    mgr = LBM_Manager(ctx, case, storage, schedule=schedule or ("phases" if storage == "f64" else "fused"),
                      scaling=scaling, storage_shift=storage_shift, interface_time=interface_time)
    mgr.fluidSimulate(req.coarse_steps())
    ctx.synchronize()
    cd, cl = drag_lift(mgr, req)
    dt = time.perf_counter() - t
    finite = True
    if with_status:
        try:
            mgr.status()
        except MTError:
            finite = False
    mgr.close()
    return (cd, cl, dt, finite) if with_status else (cd, cl, dt)


def plain_solve_seconds(ctx, cache: TemplateCache, req: Request, sample: int = 8) -> float:
    """Wall time of one request solved alone in the plain form (FP64, the
    reference's phase order): set-up, then 1/`sample` of its coarse steps
    (at least 2) timed and scaled to all of them (the per-step cost of a
    case is constant)."""
    from .lbm import LBM_Manager
    case = request_case(req, cache.get(req))
    t = time.perf_counter()
    mgr = LBM_Manager(ctx, case, "f64", schedule="phases", scaling="standard", interface_time=INTERFACE_TIME)
    ctx.synchronize()
    t_build = time.perf_counter() - t
    k = max(2, req.coarse_steps() // sample)
    t = time.perf_counter()
    mgr.fluidSimulate(k)
    ctx.synchronize()
    per = (time.perf_counter() - t) / k
    mgr.close()
    return t_build + per * req.coarse_steps()
