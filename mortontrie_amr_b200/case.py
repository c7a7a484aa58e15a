"""Flow-case parameters and the seeded synthetic cases the tests and the
benchmark use.

A case is a mesh (index sets, see mesh.py) plus the physics switches that
the reference hard-codes in LBM_Manager's constructor
(LBM_Manager.cpp:38-80) and in its compile-time constants
(header/Constants.h:164-236).
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .lattice import directions, reference_units, weights
from .mesh import Mesh, MeshSpec, Octree, Sphere, build_mesh, spec_mesh, sphere_markers

COLLISIONS = {"LBGK": 0, "Cumulant": 1}
IB_METHODS = {"DW": 0, "FH": 1, "DF": 2}
BC_MODES = {"neq": 0, "zouhe_outflow": 1, "zouhe_hh": 2}
STREAM_CONVENTIONS = {"reference": 0, "textbook": 1}
STORAGE = {"f64": 0, "f32": 1, "f16": 2, "bf16": 3}


@dataclass
class CaseParams:
    q: int = 19
    collision: str = "LBGK"
    ib_method: str = "FH"
    bc_mode: str = "neq"
    stream_convention: str = "reference"
    nu: float = 0.02                 # level-0 lattice viscosity
    u_bc: tuple = (0.05, 0.0, 0.0)   # boundary velocity (lattice units)
    u_ref: float = 0.05              # reference velocity of the unit conversion
    rho0: float = 1.0
    storage: str = "f64"
    tau: list = field(default_factory=list)
    face_u: dict = field(default_factory=dict)  # face (0..5 = W E S N B T) -> boundary velocity, else u_bc

    def taus(self, max_level: int) -> list:
        if self.tau:
            return list(self.tau)
        t, _, _ = reference_units(self.nu, self.u_ref, max_level,
                                  collision="LBGK")
        return t


@dataclass
class Case:
    mesh: Mesh
    params: CaseParams

    @property
    def max_level(self) -> int:
        return self.mesh.spec.max_level

    @property
    def q(self) -> int:
        return self.params.q


def _mesh(spec: MeshSpec, where: str):
    """The host mesher's sets ("host") or the spec alone, classified on the
    device when the case is created ("device")."""
    if where == "host":
        return build_mesh(spec)
    if where == "device":
        return spec_mesh(spec)
    raise ValueError(f"mesh must be 'host' or 'device', not {where!r}")


def sphere_case(q=19, collision="LBGK", coarse=(64, 32, 32), max_level=1, refine=None, center=(16, 16, 16),
                radius=4.0, u=0.05, re=20.0, boundary=("bc", "periodic", "periodic"), bc_mode="zouhe_outflow",
                ib_method="FH", stream_convention="reference", mesh="host", octree=None) -> Case:
    """Flow past a sphere; nu = u * 2R / Re in coarse units.  octree (an
    mesh.Octree) refines around the sphere itself instead of in boxes."""
    if octree is not None:
        refine = []
    elif refine is None:
        refine = [((4, 8, 8), (28, 24, 24))]
    nu = u * 2.0 * radius / re
    spec = MeshSpec(q=q, max_level=max_level, coarse=tuple(coarse), refine=list(refine), boundary=tuple(boundary),
                    sphere=Sphere(tuple(center), radius), octree=octree)
    p = CaseParams(q=q, collision=collision, ib_method=ib_method, bc_mode=bc_mode, nu=nu, u_bc=(u, 0.0, 0.0),
                   u_ref=u, stream_convention=stream_convention)
    return Case(_mesh(spec, mesh), p)


def surface_case(surface, q=19, collision="LBGK", coarse=(32, 16, 16), max_level=1, refine=None, ref_length=None,
                 u=0.05, re=20.0, boundary=("bc", "periodic", "periodic"), bc_mode="zouhe_outflow", ib_method="FH",
                 stream_convention="reference", mesh="host", octree=None) -> Case:
    """Flow past a closed triangulated body (an STL surface, (n, 3, 3) in
    coarse-cell units), voxelised on the finest level; nu = u * ref_length /
    Re with ref_length the body's largest extent across the flow (y, z) by
    default.  octree (an mesh.Octree) refines around the body itself
    instead of in boxes."""
    surface = np.asarray(surface, np.float64)
    if octree is not None:
        refine = []
    elif refine is None:
        lo, hi = surface.reshape(-1, 3).min(axis=0), surface.reshape(-1, 3).max(axis=0)
        refine = [(tuple(int(np.floor(v)) - 3 for v in lo), tuple(int(np.ceil(v)) + 3 for v in hi))]
    if ref_length is None:
        ext = surface.reshape(-1, 3).max(axis=0) - surface.reshape(-1, 3).min(axis=0)
        ref_length = float(max(ext[1], ext[2]))
    nu = u * ref_length / re
    spec = MeshSpec(q=q, max_level=max_level, coarse=tuple(coarse), refine=list(refine), boundary=tuple(boundary),
                    surface=surface, octree=octree)
    p = CaseParams(q=q, collision=collision, ib_method=ib_method, bc_mode=bc_mode, nu=nu, u_bc=(u, 0.0, 0.0),
                   u_ref=u, stream_convention=stream_convention)
    return Case(_mesh(spec, mesh), p)


def nested_sphere_case(q=27, collision="Cumulant", coarse=(192, 96, 96), max_level=3, center=(64, 48, 48),
                       radius=6.0, half_widths=(4.0, 2.5, 1.75), u=0.04, re=200.0,
                       boundary=("bc", "periodic", "periodic"), bc_mode="zouhe_outflow", ib_method="FH",
                       stream_convention="reference", mesh="host") -> Case:
    """Flow past a sphere refined in nested boxes centred on it: the box
    refined from level l to l+1 has half-width half_widths[l] * radius in
    coarse units (the defaults are the 4-level D3Q27 cumulant sphere case:
    192x96x96 coarse cells, R = 6 coarse = 48 finest cells, Re 200,
    inlet u 0.04, outflow, periodic lateral sides)."""
    refine = []
    for l in range(max_level):
        s = 1 << l
        hw = int(round(half_widths[l] * radius * s))
        c = [int(round(ci * s)) for ci in center]
        refine.append((tuple(ci - hw for ci in c), tuple(ci + hw for ci in c)))
    return sphere_case(q=q, collision=collision, coarse=coarse, max_level=max_level, refine=refine, center=center,
                       radius=radius, u=u, re=re, boundary=boundary, bc_mode=bc_mode, ib_method=ib_method,
                       stream_convention=stream_convention, mesh=mesh)


def cavity_case(q=19, collision="LBGK", coarse=(32, 32, 32), max_level=1, re=100.0, u_lid=0.05,
                refine=None, ib_method="FH", mesh="host") -> Case:
    """Lid-driven cavity: walls on every face (non-equilibrium boundary),
    the Top face moving at u_lid along x; nu = u_lid * nz / Re in coarse
    units.  With max_level > 0 the levels refine nested boxes under the lid
    (default: 2 coarse cells clear of the side walls, the upper quarter of
    the cavity, each finer box 2 coarse cells inside the previous one)."""
    nx, ny, nz = coarse
    nu = u_lid * nz / re
    if refine is None:
        refine = []
        lo, hi = [2, 2, nz - nz // 4 - 2], [nx - 2, ny - 2, nz - 2]
        for l in range(max_level):
            s = 1 << l
            refine.append((tuple(v * s for v in lo), tuple(v * s for v in hi)))
            lo = [v + 2 for v in lo]
            hi = [v - 2 for v in hi]
    spec = MeshSpec(q=q, max_level=max_level, coarse=tuple(coarse), refine=list(refine) if max_level else [None],
                    boundary=("bc", "bc", "bc"), sphere=None)
    if max_level == 0:
        spec = MeshSpec(q=q, max_level=1, coarse=tuple(coarse), refine=[None], boundary=("bc", "bc", "bc"))
    p = CaseParams(q=q, collision=collision, ib_method=ib_method, bc_mode="neq", nu=nu, u_bc=(0.0, 0.0, 0.0),
                   u_ref=u_lid, face_u={5: (u_lid, 0.0, 0.0)})
    return Case(_mesh(spec, mesh), p)


def df_sphere_case(radius=4, max_level=2, re=100.0, oscillating=False, u=0.05, q=19, period=2000,
                   amplitude=0.5, band_slack=0.0, mesh="host", window=None, octree=None) -> Case:
    """Flow past a sphere represented by direct-forcing Lagrangian markers
    (one per finest cell^2 of surface, 3-point kernel): coarse channel
    16R x 8R x 8R, inlet on West, outflow on East, periodic sides, centre at
    (4R, 4R, 4R), nested refinement boxes around the sphere and its path
    (transverse oscillation of `amplitude` R along y with `period` finest
    steps when oscillating), nu = u 2R / Re in coarse units, D3Q19 LBGK.
    window = (y_lo, y_hi): the boxes and the forcing band cover only the
    centre displacements in [y_lo, y_hi] (coarse cells) of the path, for a
    refinement that moves with the body (the markers still follow the whole
    path).  octree (an mesh.Octree): refine around the forcing band and its
    path instead of boxes (the fluid inside the sphere on coarser levels)."""
    r = int(radius)
    nx, ny, nz = 16 * r, 8 * r, 8 * r
    c0 = (4 * r, 4 * r, 4 * r)
    amp = amplitude * r if oscillating else 0.0
    if window is not None:
        mid, half = 0.5 * (window[0] + window[1]), 0.5 * (window[1] - window[0])
        c = (c0[0], c0[1] + mid, c0[2])
    else:
        c, half = c0, amp
    # finest box: the band (2.7 finest cells) plus the C2F shell and a margin
    mg = max(0.5 * r, 6.0 / (1 << max_level) + 0.5)
    hw = [r + mg, r + half + mg, r + mg]
    boxes = []
    for _ in range(max_level):
        boxes.append(list(hw))
        hw = [hw[0] + max(2.0, 0.5 * r), min(hw[1] + max(2.0, 0.5 * r), min(c[1], ny - c[1]) - 1.0),
              min(hw[2] + max(2.0, 0.5 * r), 4 * r - 1.0)]
    boxes = boxes[::-1]  # level 0 box first
    refine = []
    for l, b in enumerate(boxes):
        s = 1 << l
        refine.append((tuple(int(np.floor((c[a] - b[a]) * s)) for a in range(3)),
                       tuple(int(np.ceil((c[a] + b[a]) * s)) for a in range(3))))
    if octree is not None:
        # refinement made from the forcing band over the path instead of boxes
        if window is not None:
            raise ValueError("a moving window takes refinement boxes")
        refine = []
    nu = u * 2.0 * r / re
    p = CaseParams(q=q, collision="LBGK", ib_method="DF", bc_mode="zouhe_outflow", nu=nu, u_bc=(u, 0.0, 0.0),
                   u_ref=u)
    if window is not None:
        # the band of the window (its displacements as a symmetric sweep
        # about its middle); the markers of the whole path about c0
        spec = MeshSpec(q=q, max_level=max_level, coarse=(nx, ny, nz), refine=refine,
                        boundary=("bc", "periodic", "periodic"), sphere=Sphere(c, float(r)), ib="markers",
                        oscillation=(half, period), band_slack=band_slack)
        path_spec = MeshSpec(q=q, max_level=max_level, coarse=(nx, ny, nz), refine=refine,
                             boundary=spec.boundary, sphere=Sphere(c0, float(r)), ib="markers",
                             oscillation=(amp, period) if oscillating else None)
        m = _mesh(spec, mesh)
        return Case(dataclasses.replace(m, markers=sphere_markers(path_spec)), p)
    spec = MeshSpec(q=q, max_level=max_level, coarse=(nx, ny, nz), refine=refine,
                    boundary=("bc", "periodic", "periodic"), sphere=Sphere(c, float(r)), ib="markers",
                    oscillation=(amp, period) if oscillating else None, band_slack=band_slack, octree=octree)
    return Case(_mesh(spec, mesh), p)


def uniform_box_case(q=19, n=(16, 16, 16), nu=1.0 / 30.0, boundary=("periodic",) * 3, collision="LBGK",
                     u_ref=0.02, storage="f64", stream_convention="reference", empty_levels=0,
                     u_bc=(0.0, 0.0, 0.0), mesh="host") -> Case:
    """Single populated level; `empty_levels` adds empty finer levels so the
    reference harness (which needs at least two levels) can run it."""
    spec = MeshSpec(q=q, max_level=empty_levels, coarse=tuple(n), refine=[None] * empty_levels,
                    boundary=tuple(boundary))
    p = CaseParams(q=q, collision=collision, nu=nu, u_bc=tuple(u_bc), u_ref=u_ref, bc_mode="neq",
                   storage=storage, stream_convention=stream_convention)
    return Case(_mesh(spec, mesh), p)


def taylor_green_fields(n, u0=0.02, rho_amp=True):
    """TGV initial field on an n^3 periodic box with wavenumber 2 pi / n:
    u = u0 sin kx cos ky cos kz, v = -u0 cos kx sin ky cos kz, w = 0, and the
    matching pressure term in the density (c_s^2 = 1/3)."""
    nx, ny, nz = n
    k = 2.0 * np.pi / nx
    x = (np.arange(nx) + 0.5) * k
    y = (np.arange(ny) + 0.5) * (2.0 * np.pi / ny)
    z = (np.arange(nz) + 0.5) * (2.0 * np.pi / nz)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    u = u0 * np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -u0 * np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    rho = np.ones_like(u)
    if rho_amp:
        rho = rho + 3.0 * (u0 * u0 / 16.0) * (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0)
    return rho, u, v, w


def equilibrium(q, rho, ux, uy, uz):
    """BGK equilibrium, same expression order as LBM_Manager::calculateFeq
    (LBM_Manager.cpp:137-169); arrays broadcast, output shape (Q, ...)."""
    ex, ey, ez, _ = directions(q)
    w = weights(q)
    uu = ux * ux + uy * uy + uz * uz
    out = []
    for i in range(q):
        euv = ex[i] * ux + ey[i] * uy + ez[i] * uz
        out.append(rho * w[i] * (1. + 3. * euv + 4.5 * euv * euv - 1.5 * uu))
    return np.stack(out)


def perturbed_populations(case: Case, seed: int = 1234, amp: float = 0.02):
    """Seeded near-equilibrium populations for every stored cell of every
    level (f = feq(rho, u) * (1 + amp * noise), rho in [0.95, 1.05],
    |u| < 0.05), keyed by the sorted cell keys.  Solid cells stay zero."""
    rng = np.random.default_rng(seed)
    out = []
    for l in range(case.max_level + 1):
        keys = case.mesh.all_keys(l)
        n = keys.size
        rho = rng.uniform(0.95, 1.05, n)
        u = rng.uniform(-0.03, 0.03, (3, n))
        f = equilibrium(case.q, rho, u[0], u[1], u[2]) * (1.0 + amp * rng.uniform(-1, 1, (case.q, n)))
        if l == case.max_level and case.mesh.levels[l]["lat_sf"].size:
            sf = np.isin(keys, case.mesh.levels[l]["lat_sf"])
            f[:, sf] = 0.0
        out.append((keys, np.ascontiguousarray(f)))
    return out
