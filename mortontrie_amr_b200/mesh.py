"""Box-refinement mesher that emits the reference's lattice index-set contract.

The reference builds its per-level index sets in Lat_Manager::voxelize
(Lat_Voxelize.cpp:17-733) from an STL-driven octree.  The LBM step only
consumes the resulting sets (Lat_Manager.hpp:245-316):

  lat_f[l]              cells that collide and stream
  lat_overlap_F2C[l]    coarse cells under the fine region's outer shell:
                        collide, receive f by coalescence, never stream
  lat_overlap_C2F[l]    fine cells that are children of F2C[l-1]: their fcol
                        is copied from f, then overwritten by explosion
  ghost_overlap_C2F[l]  fine cells just outside the fine region that give
                        C2F cells something to pull from
  ghost_overlap_F2C[l]  coarse lat_f neighbours of F2C cells (explosion
                        sources for ghost_overlap_C2F)
  lat_sf                finest-level solid cells (f = fcol = 0 storage)
  lat_bc[26]            level-0 boundary shell split into 6 faces, 12 edges,
                        8 corners (Lat_Voxelize.cpp:242-288)
  dis                   finest-level cells with at least one link that
                        crosses the solid: normalised wall distance per
                        direction q>=1, -1 where the link is free
                        (Lat_Voxelize.cpp:1252-1285)

This module re-creates that contract for nested refinement boxes and an
analytic sphere, which is what the flow cases here need.  The sets it
returns are plain sorted uint64 key arrays.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .lattice import cell_key, directions

SET_NAMES = ("lat_f", "overlap_F2C", "overlap_C2F", "ghost_overlap_C2F", "ghost_overlap_F2C", "lat_sf")

# lat_bc index -> side of the box on each axis (-1 low, +1 high, 0 none);
# the index order is the reference's Bdry_Type enum (D3Q19_BC_Manager.hpp:25-53).
BC_SIDES = [
    (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1),
    (1, 1, 0), (-1, 1, 0), (-1, -1, 0), (1, -1, 0),
    (0, 1, 1), (0, -1, 1), (0, 1, -1), (0, -1, -1),
    (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1),
    (1, 1, 1), (-1, 1, 1), (-1, -1, 1), (1, -1, 1),
    (1, 1, -1), (-1, 1, -1), (-1, -1, -1), (1, -1, -1),
]


@dataclass
class Sphere:
    center: tuple  # coarse-cell units, measured from the box corner
    radius: float  # coarse-cell units


@dataclass
class MeshSpec:
    q: int
    max_level: int
    coarse: tuple                      # (nx, ny, nz) coarse cells
    # per level l < L: ((lo), (hi)) in level-l cells, or None for an empty
    # finer level (the reference cannot run with a single level: its
    # LBM_Manager::defineRunOrder indexes past the level array when
    # C_max_level == 0, LBM_Manager.cpp:105-128)
    refine: list = field(default_factory=list)
    boundary: tuple = ("bc", "bc", "bc")  # per axis: "bc" (level-0 boundary shell) or "periodic"
    sphere: Optional[Sphere] = None
    # "links": voxelised solid + wall distances (the reference's
    # SinglePointInterpolation); "markers": direct forcing on Lagrangian
    # surface markers, fluid inside the sphere and a forcing band
    ib: str = "links"
    # transverse oscillation of a marker sphere: (amplitude in coarse cells,
    # period in finest steps), along y
    oscillation: Optional[tuple] = None
    # extra inner depth of the forcing band in coarse cells, so that one mesh
    # serves marker spheres of radius in [radius - band_slack, radius]
    band_slack: float = 0.0
    # closed triangulated solid surface (n, 3, 3) in coarse-cell units,
    # voxelised on the finest level instead of a sphere (links mode)
    surface: Optional[np.ndarray] = None
    # refinement driven by the body instead of boxes (refine then lists no
    # boxes): see Octree
    octree: Optional["Octree"] = None


@dataclass
class Octree:
    """Refinement regions made from the body (sphere or surface) instead of
    boxes: the finest level covers every level-(L-1) cell within `band` of
    those cells of the body's surface and inside it (the near-solid cells
    Grid_Manager::generate_inner refines, Grid_Manager.cpp:136-454; for a
    direct-forcing sphere the cells within `band` of its forcing band over
    the whole path, the fluid inside left to coarser levels), and
    every coarser level covers the next finer region grown by `margin` of
    its own cells, rounded out to whole parent cells (the intermediate
    levels the reference's generate_intermediate would make and leaves
    empty, Grid_Manager.cpp:99-102).  The levels nest 2:1 by construction."""
    band: float = 3.0   # level-(L-1) cells around the surface
    margin: int = 4     # level-l cells between level l+1's region and level l's edge


@dataclass
class Markers:
    """Lagrangian markers of a direct-forcing sphere, finest-level cell units."""
    ref: np.ndarray     # (3, nm) offsets from the centre
    dv: np.ndarray      # (nm,) volume weight of each marker
    center: tuple       # initial centre
    path: np.ndarray    # (period, 6): centre displacement and velocity at substep t % period


def sphere_markers(spec: "MeshSpec", radius: Optional[float] = None) -> Markers:
    """One marker per finest cell^2 of surface on a Fibonacci lattice; the
    path samples y(t) = A sin(2 pi t / T) and its velocity per finest step.
    radius (coarse cells) defaults to the mesh's sphere radius."""
    L = spec.max_level
    s = 1 << L
    r = (spec.sphere.radius if radius is None else radius) * s
    nm = max(1, int(round(4.0 * np.pi * r * r)))
    i = np.arange(nm) + 0.5
    zc = 1.0 - 2.0 * i / nm
    rc = np.sqrt(np.maximum(0.0, 1.0 - zc * zc))
    phi = i * (np.pi * (3.0 - np.sqrt(5.0)))
    ref = np.stack([r * rc * np.cos(phi), r * rc * np.sin(phi), r * zc])
    dv = np.full(nm, 4.0 * np.pi * r * r / nm)
    center = tuple(float(c * s) for c in spec.sphere.center)
    if spec.oscillation:
        amp, period = spec.oscillation[0] * s, int(spec.oscillation[1])
        t = np.arange(period)
        path = np.zeros((period, 6))
        path[:, 1] = amp * np.sin(2.0 * np.pi * t / period)
        path[:, 4] = amp * (2.0 * np.pi / period) * np.cos(2.0 * np.pi * t / period)
    else:
        path = np.zeros((1, 6))
    return Markers(ref=np.ascontiguousarray(ref), dv=dv, center=center, path=np.ascontiguousarray(path))


@dataclass
class Mesh:
    spec: MeshSpec
    levels: list          # per level: dict set name -> sorted uint64 keys
    lat_bc: list          # 26 sorted uint64 key arrays (level 0)
    dis_keys: np.ndarray  # sorted finest-level keys
    dis_rows: np.ndarray  # (n, Q-1) float64
    extent: list          # per level: (nx, ny, nz) in that level's cells
    markers: Optional["Markers"] = None

    def all_keys(self, level: int) -> np.ndarray:
        parts = [self.levels[level][s] for s in SET_NAMES]
        if level == 0:
            parts += list(self.lat_bc)
        return _sorted_unique(np.concatenate(parts)) if parts else np.zeros(0, np.uint64)

    def n_cells(self) -> list:
        return [int(self.all_keys(l).size) for l in range(self.spec.max_level + 1)]


@dataclass
class SpecMesh:
    """A mesh known by its spec only: the device classifies the lattice when
    the case is created (mt_case_generate), producing the sets build_mesh
    would; the markers of a direct-forcing sphere are made on the host."""
    spec: MeshSpec
    markers: Optional["Markers"] = None


def spec_mesh(spec: MeshSpec) -> SpecMesh:
    if spec.octree is not None:
        if spec.refine:
            raise ValueError("refinement boxes and an octree are exclusive")
        octree_regions(spec)  # the regions' own checks, before the device build
        mk = sphere_markers(spec) if (spec.sphere is not None and spec.ib == "markers") else None
        return SpecMesh(spec=spec, markers=mk)
    if len(spec.refine) != spec.max_level:
        raise ValueError("need one refinement box per level below the maximum level")
    mk = sphere_markers(spec) if (spec.sphere is not None and spec.ib == "markers") else None
    return SpecMesh(spec=spec, markers=mk)


def estimate_cells(spec: MeshSpec) -> list:
    """Upper bound of the stored cells per level from the boxes alone (no
    classification): the level's box minus the interior under the next
    refinement box, plus a one-cell layer outside the box (ghost C2F) and
    outside the refinement box (ghost F2C); for an octree, each level's
    domain and its one-cell layer."""
    def vol(lo, hi, g=0):
        return int(np.prod([max(0, h - l + 2 * g) for l, h in zip(lo, hi)]))
    if spec.octree is not None:
        # each level's domain (the children of its region) with its ghost layer
        regions = octree_regions(spec)
        out = [vol((0, 0, 0), tuple(spec.coarse))]
        for l in range(1, spec.max_level + 1):
            out.append(int(regions[l].children().dilate(1).mask.sum()))
        return out
    out = []
    lo, hi = (0, 0, 0), tuple(spec.coarse)
    for l in range(spec.max_level + 1):
        if vol(lo, hi) == 0:
            out.append(0)
            continue
        n = vol(lo, hi) + (vol(lo, hi, 1) - vol(lo, hi) if l > 0 else 0)
        box = spec.refine[l] if l < spec.max_level else None
        if box is not None:
            n -= vol(box[0], box[1], -1)
            n += vol(box[0], box[1], 1) - vol(box[0], box[1])
            lo, hi = tuple(2 * v for v in box[0]), tuple(2 * v for v in box[1])
        else:
            lo, hi = (0, 0, 0), (0, 0, 0)
        out.append(n)
    return out


class Region:
    """A set of cells of one level as a dense mask over its bounding box:
    cell (x, y, z) is in the set iff mask[x - lo[0], y - lo[1], z - lo[2]]."""

    def __init__(self, lo, mask):
        self.lo = np.asarray(lo, np.int64)
        self.mask = np.ascontiguousarray(mask, bool)

    @property
    def hi(self):
        return self.lo + np.array(self.mask.shape, np.int64)

    def padded(self, p):
        return Region(self.lo - p, np.pad(self.mask, p))

    def dilate(self, m):
        """Every cell within Chebyshev distance m of the set (a cube of
        half-width m, one axis at a time)."""
        r = self.padded(m)
        mk = r.mask
        for axis in range(3):
            acc = mk.copy()
            for d in range(1, m + 1):
                acc |= _shifted(mk, d, axis)
                acc |= _shifted(mk, -d, axis)
            mk = acc
        return Region(r.lo, mk)

    def shell(self):
        """Cells of the set with one of their 26 neighbours outside it (the
        set minus its erosion by the 3x3x3 cube, one axis at a time)."""
        r = self.padded(1)
        er = r.mask
        for axis in range(3):
            er = er & _shifted(er, 1, axis) & _shifted(er, -1, axis)
        return Region(r.lo, r.mask & ~er)

    def parents(self):
        """The level-(l-1) cells with at least one child in the set."""
        lo = self.lo - (self.lo & 1)
        pre = self.lo - lo
        shape = np.array(self.mask.shape) + pre
        post = shape & 1
        m = np.pad(self.mask, [(int(a), int(b)) for a, b in zip(pre, post)])
        nx, ny, nz = (np.array(m.shape) // 2).tolist()
        return Region(lo // 2, m.reshape(nx, 2, ny, 2, nz, 2).any(axis=(1, 3, 5)))

    def children(self):
        """The level-(l+1) cells whose parent is in the set."""
        m = self.mask.repeat(2, axis=0).repeat(2, axis=1).repeat(2, axis=2)
        return Region(2 * self.lo, m)

    def contains(self, x, y, z):
        x, y, z = (np.asarray(v, np.int64) for v in (x, y, z))
        ix, iy, iz = x - self.lo[0], y - self.lo[1], z - self.lo[2]
        sh = self.mask.shape
        ok = (ix >= 0) & (ix < sh[0]) & (iy >= 0) & (iy < sh[1]) & (iz >= 0) & (iz < sh[2])
        out = np.zeros(x.size, bool)
        out[ok] = self.mask[ix[ok], iy[ok], iz[ok]]
        return out

    def cells(self):
        ix, iy, iz = np.nonzero(self.mask)
        return ix + self.lo[0], iy + self.lo[1], iz + self.lo[2]


def _shifted(m, d, axis):
    """m moved by d cells along axis: out[c] = m[c - d], False where c - d
    falls outside."""
    out = np.zeros_like(m)
    src = [slice(None)] * 3
    dst = [slice(None)] * 3
    if d > 0:
        src[axis], dst[axis] = slice(0, -d), slice(d, None)
    else:
        src[axis], dst[axis] = slice(-d, None), slice(0, d)
    out[tuple(dst)] = m[tuple(src)]
    return out


def box_region(lo, hi):
    return Region(lo, np.ones(tuple(int(h - l) for l, h in zip(lo, hi)), bool))


def surface_points(tris, spacing):
    """Points on every triangle no further apart than `spacing` (a
    barycentric lattice per triangle, vertices included)."""
    tris = np.asarray(tris, np.float64)
    out = []
    for t in tris:
        e = max(np.linalg.norm(t[1] - t[0]), np.linalg.norm(t[2] - t[0]), np.linalg.norm(t[2] - t[1]))
        n = max(1, int(np.ceil(e / spacing)))
        i, j = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
        keep = (i + j) <= n
        a, b = i[keep] / n, j[keep] / n
        out.append(t[0] + a[:, None] * (t[1] - t[0]) + b[:, None] * (t[2] - t[0]))
    return np.concatenate(out) if out else np.zeros((0, 3))


def octree_regions(spec: "MeshSpec") -> list:
    """regions[l] for l = 1..L: the level-(l-1) cells refined to level l
    (regions[0] is None), made from the body as Octree describes."""
    L = spec.max_level
    oc = spec.octree
    if L < 1:
        raise ValueError("an octree needs a refined level")
    lv = L - 1
    s = float(1 << lv)
    band = float(oc.band)
    if spec.surface is not None:
        tris = np.asarray(spec.surface, np.float64) * s
        pts = surface_points(tris, 0.5)
        lo = np.floor(pts.min(axis=0)).astype(np.int64) - int(np.ceil(band)) - 1
        hi = np.floor(pts.max(axis=0)).astype(np.int64) + int(np.ceil(band)) + 2
        mask = np.zeros(tuple((hi - lo).tolist()), bool)
        c = np.floor(pts).astype(np.int64) - lo
        mask[c[:, 0], c[:, 1], c[:, 2]] = True
        near = Region(lo, mask).dilate(int(np.ceil(band)))
        gx, gy, gz = _grid(near.lo, near.hi)
        inside = surface_inside(tris, gx, gy, gz).reshape(near.mask.shape)
        fine = Region(near.lo, near.mask | inside)
    elif spec.sphere is not None and spec.ib == "markers":
        # a direct-forcing sphere: only the forcing band over the whole path
        # (finest cells within 2.7 of the surface at some position, and
        # band_slack deeper; 1.35 level-(L-1) cells) and `band` around it; the
        # fluid inside stays on coarser levels
        c = np.asarray(spec.sphere.center, np.float64) * s
        r = spec.sphere.radius * s
        amp = spec.oscillation[0] * s if spec.oscillation else 0.0
        slack = spec.band_slack * s
        reach = band + np.sqrt(3.0) / 2.0
        ext = np.array([r, r + amp, r]) + 1.35 + reach + 1.0
        lo = np.floor(c - ext).astype(np.int64) - 1
        hi = np.ceil(c + ext).astype(np.int64) + 1
        gx, gy, gz = _grid(lo, hi)
        px, py, pz = gx + 0.5 - c[0], gy + 0.5 - c[1], gz + 0.5 - c[2]
        qy = np.clip(py, -amp, amp)
        dmin = np.sqrt(px * px + (py - qy) ** 2 + pz * pz)
        dmax = np.sqrt(px * px + (np.abs(py) + amp) ** 2 + pz * pz)
        keep = (dmin <= r + 1.35 + reach) & (dmax >= r - 1.35 - slack - reach)
        fine = Region(lo, keep.reshape(tuple((hi - lo).tolist())))
    elif spec.sphere is not None:
        c = np.asarray(spec.sphere.center, np.float64) * s
        r = spec.sphere.radius * s
        ext = r + band + 1.0
        lo = np.floor(c - ext).astype(np.int64) - 1
        hi = np.ceil(c + ext).astype(np.int64) + 1
        gx, gy, gz = _grid(lo, hi)
        d = np.sqrt((gx + 0.5 - c[0]) ** 2 + (gy + 0.5 - c[1]) ** 2 + (gz + 0.5 - c[2]) ** 2)
        # every cell that reaches within `band` of the surface, and the inside
        fine = Region(lo, (d <= r + band + np.sqrt(3.0) / 2.0).reshape(tuple((hi - lo).tolist())))
    else:
        raise ValueError("an octree is made from a body: a sphere or a surface")
    regions = [None] * (L + 1)
    regions[L] = fine
    for l in range(L - 1, 0, -1):
        regions[l] = regions[l + 1].dilate(int(oc.margin)).parents()
    for l in range(1, L + 1):
        ext = np.array(spec.coarse, np.int64) << (l - 1)
        x, y, z = regions[l].cells()
        if x.size == 0:
            raise ValueError(f"level {l}: empty octree region")
        if (x.min() < 0 or y.min() < 0 or z.min() < 0 or x.max() >= ext[0] or y.max() >= ext[1]
                or z.max() >= ext[2]):
            raise ValueError(f"level {l}: the octree region leaves the domain (a larger box or a smaller margin)")
    return regions


def _grid(lo, hi):
    xs = np.arange(lo[0], hi[0], dtype=np.int64)
    ys = np.arange(lo[1], hi[1], dtype=np.int64)
    zs = np.arange(lo[2], hi[2], dtype=np.int64)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    return X.ravel(), Y.ravel(), Z.ravel()


def _shell_mask(x, y, z, lo, hi, width):
    return ((x < lo[0] + width) | (x >= hi[0] - width) | (y < lo[1] + width) | (y >= hi[1] - width)
            | (z < lo[2] + width) | (z >= hi[2] - width))


def _inside(x, y, z, lo, hi):
    return ((x >= lo[0]) & (x < hi[0]) & (y >= lo[1]) & (y < hi[1]) & (z >= lo[2]) & (z < hi[2]))


def _neighbours(x, y, z, q, extent, periodic):
    """Q-1 neighbour coordinates, wrapped on periodic axes."""
    ex, ey, ez, _ = directions(q)
    out = []
    for d in range(1, q):
        nx_, ny_, nz_ = x + ex[d], y + ey[d], z + ez[d]
        if periodic[0]:
            nx_ = np.mod(nx_, extent[0])
        if periodic[1]:
            ny_ = np.mod(ny_, extent[1])
        if periodic[2]:
            nz_ = np.mod(nz_, extent[2])
        out.append((nx_, ny_, nz_))
    return out


def _sorted_unique(a):
    a = np.sort(np.asarray(a, np.uint64))
    if a.size < 2:
        return a
    keep = np.empty(a.size, bool)
    keep[0] = True
    np.not_equal(a[1:], a[:-1], out=keep[1:])
    return a[keep]


def _in_sorted(a, sorted_b):
    """Membership of each key of a in the sorted unique array sorted_b."""
    a = np.asarray(a, np.uint64)
    if sorted_b.size == 0 or a.size == 0:
        return np.zeros(a.size, bool)
    idx = np.searchsorted(sorted_b, a)
    np.minimum(idx, sorted_b.size - 1, out=idx)
    return sorted_b[idx] == a


def build_mesh(spec: MeshSpec) -> Mesh:
    L = spec.max_level
    q = spec.q
    octree = spec.octree is not None
    if octree:
        if spec.refine:
            raise ValueError("refinement boxes and an octree are exclusive")
    elif len(spec.refine) != L:
        raise ValueError("need one refinement box per level below the maximum level")
    periodic = tuple(b == "periodic" for b in spec.boundary)
    nx, ny, nz = spec.coarse
    levels = []
    extents = []
    lat_bc = [np.zeros(0, np.uint64) for _ in range(26)]

    # domain of each level in its own cell units: a box, or for an octree
    # the children of the level's region
    dom_lo = [(0, 0, 0)]
    dom_hi = [(nx, ny, nz)]
    regions = octree_regions(spec) if octree else None
    if not octree:
        for l in range(L):
            if spec.refine[l] is None or dom_hi[-1] == (0, 0, 0):
                dom_lo.append((0, 0, 0))
                dom_hi.append((0, 0, 0))
                continue
            lo, hi = spec.refine[l]
            dom_lo.append(tuple(2 * v for v in lo))
            dom_hi.append(tuple(2 * v for v in hi))
    for l in range(L + 1):
        extents.append(tuple((n << l) for n in (nx, ny, nz)))

    for l in range(L + 1):
        if octree and l > 0:
            x, y, z = regions[l].children().cells()
        else:
            x, y, z = _grid(dom_lo[l], dom_hi[l])
        sets = {}
        stored = np.ones(x.size, bool)
        is_bc = np.zeros(x.size, bool)
        if l == 0:
            side = np.zeros((x.size, 3), np.int64)
            for a, (c, n) in enumerate(zip((x, y, z), (nx, ny, nz))):
                if spec.boundary[a] == "bc":
                    side[c == 0, a] = -1
                    side[c == n - 1, a] = 1
            is_bc = np.any(side != 0, axis=1)
            for i, s in enumerate(BC_SIDES):
                m = is_bc & (side[:, 0] == s[0]) & (side[:, 1] == s[1]) & (side[:, 2] == s[2])
                lat_bc[i] = _sorted_unique(cell_key(L, 0, x[m], y[m], z[m]))
        f2c = np.zeros(x.size, bool)
        if octree and l < L:
            # the region's outer layer of level-l cells; the rest of it is
            # stored on the finer level only
            inside = regions[l + 1].contains(x, y, z)
            f2c = regions[l + 1].shell().contains(x, y, z)
            stored &= ~(inside & ~f2c)
            if np.any(inside & is_bc):
                raise ValueError("the octree region touches the boundary shell")
        elif l < L and dom_hi[l + 1] != (0, 0, 0):
            lo, hi = spec.refine[l]
            inside = _inside(x, y, z, lo, hi)
            f2c = inside & _shell_mask(x, y, z, lo, hi, 1)
            stored &= ~(inside & ~f2c)
            if np.any(inside & is_bc):
                raise ValueError("refinement box touches the boundary shell")
        c2f = np.zeros(x.size, bool)
        if l > 0:
            # the children of the coarser level's F2C cells: for a box, the
            # two-cell shell of the level's domain
            c2f = (regions[l].shell().children().contains(x, y, z) if octree
                   else _shell_mask(x, y, z, dom_lo[l], dom_hi[l], 2))
            if np.any(c2f & f2c):
                raise ValueError(f"level {l}: refinement {'region' if octree else 'box'} too close to the "
                                 "coarse/fine interface")
        fluid = stored & ~is_bc & ~f2c & ~c2f
        sets["overlap_F2C"] = _sorted_unique(cell_key(L, l, x[f2c], y[f2c], z[f2c]))
        sets["overlap_C2F"] = _sorted_unique(cell_key(L, l, x[c2f], y[c2f], z[c2f]))
        sets["lat_sf"] = np.zeros(0, np.uint64)
        fx, fy, fz = x[fluid], y[fluid], z[fluid]
        if l == L and spec.sphere is not None and spec.ib == "markers":
            # every cell a marker's 3x3x3 stencil can reach over the whole path:
            # within 1.5 sqrt(3) of the surface of some position of the sphere
            s = 1 << L
            cx, cy, cz = (c * s for c in spec.sphere.center)
            r = spec.sphere.radius * s
            amp = spec.oscillation[0] * s if spec.oscillation else 0.0
            px, py, pz = fx + 0.5 - cx, fy + 0.5 - cy, fz + 0.5 - cz
            qy = np.clip(py, -amp, amp)
            dmin = np.sqrt(px * px + (py - qy) ** 2 + pz * pz)
            dmax = np.sqrt(px * px + (np.abs(py) + amp) ** 2 + pz * pz)
            m = 2.7
            band = (dmin <= r + m) & (dmax >= r - m - spec.band_slack * s)
            sets["ib_band"] = _sorted_unique(cell_key(L, l, fx[band], fy[band], fz[band]))
        elif l == L and spec.surface is not None:
            if L == 0:
                raise ValueError("the solid boundary is only applied on a refined finest level")
            solid = surface_inside(np.asarray(spec.surface, np.float64) * float(1 << L), fx, fy, fz)
            sets["lat_sf"] = _sorted_unique(cell_key(L, l, fx[solid], fy[solid], fz[solid]))
            fx, fy, fz = fx[~solid], fy[~solid], fz[~solid]
        elif l == L and spec.sphere is not None:
            if L == 0:
                raise ValueError("the solid boundary is only applied on a refined finest level")
            s = 1 << L
            cx, cy, cz = (c * s for c in spec.sphere.center)
            r = spec.sphere.radius * s
            px, py, pz = fx + 0.5, fy + 0.5, fz + 0.5
            solid = (px - cx) ** 2 + (py - cy) ** 2 + (pz - cz) ** 2 < r * r
            # every neighbour of the solid must be a plain fluid cell
            sets["lat_sf"] = _sorted_unique(cell_key(L, l, fx[solid], fy[solid], fz[solid]))
            fx, fy, fz = fx[~solid], fy[~solid], fz[~solid]
        sets["lat_f"] = _sorted_unique(cell_key(L, l, fx, fy, fz))
        levels.append(sets)

    # ghost layers (Lat_Voxelize.cpp:676-733 semantics)
    for l in range(L + 1):
        sets = levels[l]
        if l > 0:
            cx_, cy_, cz_ = _coords_of(sets["overlap_C2F"], L, l)
            cand = []
            for (a, b, c) in _neighbours(cx_, cy_, cz_, q, extents[l], periodic):
                ok = (a >= 0) & (b >= 0) & (c >= 0)
                cand.append(cell_key(L, l, a[ok], b[ok], c[ok]))
            cand = _sorted_unique(np.concatenate(cand)) if cand else np.zeros(0, np.uint64)
            keep = ~_in_sorted(cand, sets["lat_f"]) & ~_in_sorted(cand, sets["overlap_C2F"])
            sets["ghost_overlap_C2F"] = cand[keep]
            bad = (_in_sorted(sets["ghost_overlap_C2F"], sets["overlap_F2C"])
                   | _in_sorted(sets["ghost_overlap_C2F"], sets["lat_sf"]))
            if np.any(bad):
                raise ValueError(f"level {l}: ghost layer overlaps the next interface or the solid")
        else:
            sets["ghost_overlap_C2F"] = np.zeros(0, np.uint64)
        if l < L:
            fx_, fy_, fz_ = _coords_of(sets["overlap_F2C"], L, l)
            cand = []
            for (a, b, c) in _neighbours(fx_, fy_, fz_, q, extents[l], periodic):
                ok = (a >= 0) & (b >= 0) & (c >= 0)
                cand.append(cell_key(L, l, a[ok], b[ok], c[ok]))
            cand = _sorted_unique(np.concatenate(cand)) if cand else np.zeros(0, np.uint64)
            sets["ghost_overlap_F2C"] = cand[_in_sorted(cand, sets["lat_f"])]
        else:
            sets["ghost_overlap_F2C"] = np.zeros(0, np.uint64)

    dis_keys = np.zeros(0, np.uint64)
    dis_rows = np.zeros((0, q - 1))
    markers = None
    if spec.sphere is not None and spec.ib == "markers":
        band = levels[L].get("ib_band", np.zeros(0, np.uint64))
        if np.any(_in_sorted(band, levels[L]["overlap_C2F"])) or np.any(_in_sorted(band, levels[L]["ghost_overlap_C2F"])):
            raise ValueError("the forcing band reaches the coarse/fine interface")
        bx, by, bz = _coords_of(band, L, L)
        for (a, b, c) in _neighbours(bx, by, bz, q, extents[L], periodic):
            k = cell_key(L, L, a, b, c)
            if np.any(_in_sorted(k, levels[L]["overlap_C2F"])):
                raise ValueError("the forcing band is too close to the coarse/fine interface")
        markers = sphere_markers(spec)
    elif spec.sphere is not None or spec.surface is not None:
        if spec.surface is not None:
            dis_keys, dis_rows = surface_links(np.asarray(spec.surface, np.float64) * float(1 << L), q,
                                               levels[L]["lat_f"], L)
        else:
            dis_keys, dis_rows = _sphere_links(spec, levels[L]["lat_f"])
        sf_keys = levels[L]["lat_sf"]
        # IB cells must be plain lat_f cells; the solid must stay clear of C2F.
        sx, sy, sz = _coords_of(sf_keys, L, L)
        for (a, b, c) in _neighbours(sx, sy, sz, q, extents[L], periodic):
            k = cell_key(L, L, a, b, c)
            if np.any(_in_sorted(k, levels[L]["overlap_C2F"])) or np.any(_in_sorted(k, levels[L]["ghost_overlap_C2F"])):
                raise ValueError("solid too close to the coarse/fine interface")
    return Mesh(spec=spec, levels=levels, lat_bc=lat_bc, dis_keys=dis_keys, dis_rows=dis_rows,
                extent=extents, markers=markers)


def _edge_orient(u, v, py, pz):
    """Orientation of (py, pz) against the directed edge u -> v in the (y, z)
    plane, evaluated with the endpoints in lexicographic order and negated
    when swapped, so that the two traversals of an edge give exactly
    opposite values."""
    swap = (u[0] > v[0]) | ((u[0] == v[0]) & (u[1] > v[1]))
    P0 = np.where(swap, v[0], u[0]), np.where(swap, v[1], u[1])
    R0 = np.where(swap, u[0], v[0]), np.where(swap, u[1], v[1])
    o = (R0[0] - P0[0]) * (pz - P0[1]) - (R0[1] - P0[1]) * (py - P0[0])
    return np.where(swap, -o, o)


def column_crossings(tri, ys, zs):
    """Crossings of the lines {(t, ys + 0.5, zs + 0.5)} with one triangle
    (finest-cell units): (inside mask, x of the crossing).  The projected
    triangle is taken counter-clockwise in (y, z); a line through an edge or
    a vertex belongs to the triangle when the edge is a top or left edge
    (z decreasing, or z constant and y decreasing along the counter-clockwise
    traversal), so a line through a shared edge crosses exactly one of two
    adjacent triangles and touches a silhouette edge zero or two times."""
    a, b, c = tri[0], tri[1], tri[2]
    area = (b[1] - a[1]) * (c[2] - a[2]) - (b[2] - a[2]) * (c[1] - a[1])
    py, pz = ys + 0.5, zs + 0.5
    if area == 0.0:
        return np.zeros(py.shape, bool), np.zeros(py.shape)
    verts = (a, b, c) if area > 0.0 else (a, c, b)
    inside = np.ones(py.shape, bool)
    for i in range(3):
        u, v = verts[i], verts[(i + 1) % 3]
        o = _edge_orient((u[1], u[2]), (v[1], v[2]), py, pz)
        dy, dz = v[1] - u[1], v[2] - u[2]
        top_left = (dz < 0.0) or (dz == 0.0 and dy < 0.0)
        inside &= (o > 0.0) | ((o == 0.0) & top_left)
    ny = (b[2] - a[2]) * (c[0] - a[0]) - (b[0] - a[0]) * (c[2] - a[2])
    nz = (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])
    x = a[0] - (ny * (py - a[1]) + nz * (pz - a[2])) / area
    return inside, x


def _tri_columns(tri):
    """Finest-level (y, z) columns whose centre lines may cross the triangle."""
    lo, hi = tri.min(axis=0), tri.max(axis=0)
    y0, y1 = int(np.ceil(lo[1] - 0.5)), int(np.floor(hi[1] - 0.5))
    z0, z1 = int(np.ceil(lo[2] - 0.5)), int(np.floor(hi[2] - 0.5))
    return y0, y1, z0, z1


def surface_inside(tris, fx, fy, fz):
    """Cells whose centre lies inside the closed surface (finest-cell units):
    an odd number of crossings of the +x ray from the centre (crossing x
    strictly above the centre's x)."""
    fx, fy, fz = (np.asarray(v, np.int64) for v in (fx, fy, fz))
    cols = {}
    for tri in tris:
        y0, y1, z0, z1 = _tri_columns(tri)
        if y1 < y0 or z1 < z0:
            continue
        Y, Z = np.meshgrid(np.arange(y0, y1 + 1), np.arange(z0, z1 + 1), indexing="ij")
        ins, x = column_crossings(tri, Y.ravel().astype(np.float64), Z.ravel().astype(np.float64))
        for yy, zz, xx in zip(Y.ravel()[ins].tolist(), Z.ravel()[ins].tolist(), x[ins].tolist()):
            cols.setdefault((yy, zz), []).append(xx)
    solid = np.zeros(fx.size, bool)
    if not cols:
        return solid
    key = fy * (1 << 21) + fz
    order = np.argsort(key, kind="stable")
    ks = key[order]
    for (yy, zz), xs in cols.items():
        k = yy * (1 << 21) + zz
        i0, i1 = np.searchsorted(ks, k, "left"), np.searchsorted(ks, k, "right")
        if i0 == i1:
            continue
        idx = order[i0:i1]
        xs = np.sort(np.array(xs))
        above = xs.size - np.searchsorted(xs, fx[idx] + 0.5, "right")
        solid[idx] = (above & 1) == 1
    return solid


LINK_EPS = 1e-10


def link_hits(tri, px, py, pz, q):
    """Normalised wall distance of the links of cells with centres (px, py,
    pz) across one triangle (ComplexBoundary's dis convention: 0 at the cell
    centre, 1 at the neighbour's), -1 where the link misses it.  The
    intersection is Shape::intersect_line_with_triangle (Shape.cpp:809-843:
    Moller-Trumbore on the unit link direction, the crossing point rebuilt
    from its barycentric coordinates and measured from the centre) and the
    [0, 1] filter of Lat_Manager::compute_distance (Lat_Voxelize.cpp
    :1252-1285); the barycentric bounds include the edges (>= -1e-10) so that
    a link through an edge shared by two triangles is not missed."""
    ex, ey, ez, _ = directions(q)
    v1, v2, v3 = tri[0], tri[1], tri[2]
    e1 = (v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2])
    e2 = (v3[0] - v1[0], v3[1] - v1[1], v3[2] - v1[2])
    sx, sy, sz = px - v1[0], py - v1[1], pz - v1[2]
    out = np.full((px.size, q - 1), -1.0)
    for k in range(1, q):
        gx, gy, gz = float(ex[k]), float(ey[k]), float(ez[k])
        mag = np.sqrt(gx * gx + gy * gy + gz * gz)
        dx, dy, dz = gx / mag, gy / mag, gz / mag
        s1 = (dy * e2[2] - dz * e2[1], dz * e2[0] - dx * e2[2], dx * e2[1] - dy * e2[0])
        s2 = (sy * e1[2] - sz * e1[1], sz * e1[0] - sx * e1[2], sx * e1[1] - sy * e1[0])
        s1e1 = s1[0] * e1[0] + s1[1] * e1[1] + s1[2] * e1[2]
        if s1e1 == 0.0:
            continue
        with np.errstate(divide="ignore", invalid="ignore"):
            t = (s2[0] * e2[0] + s2[1] * e2[1] + s2[2] * e2[2]) / s1e1
            b1 = (s1[0] * sx + s1[1] * sy + s1[2] * sz) / s1e1
            b2 = (s2[0] * dx + s2[1] * dy + s2[2] * dz) / s1e1
        b0 = 1.0 - b1 - b2
        ok = (t >= LINK_EPS) & (b1 >= -LINK_EPS) & (b2 >= -LINK_EPS) & (b0 >= -LINK_EPS)
        ix = b0 * v1[0] + b1 * v2[0] + b2 * v3[0]
        iy = b0 * v1[1] + b1 * v2[1] + b2 * v3[1]
        iz = b0 * v1[2] + b1 * v2[2] + b2 * v3[2]
        dist = np.sqrt((ix - px) * (ix - px) + (iy - py) * (iy - py) + (iz - pz) * (iz - pz))
        nrm = dist / mag
        ok &= (nrm >= 0.0) & (nrm <= 1.0)
        out[ok, k - 1] = nrm[ok]
    return out


def surface_links(tris, q, fluid_keys, L):
    """dis rows of the finest fluid cells whose links cross the surface: per
    link the smallest normalised distance over the triangles."""
    x, y, z = _coords_of(fluid_keys, L, L)
    rows = np.full((x.size, q - 1), -1.0)
    key = (x * (1 << 21) + y) * (1 << 21) + z
    order = np.argsort(key, kind="stable")
    ks = key[order]
    for tri in tris:
        lo, hi = tri.min(axis=0), tri.max(axis=0)
        rng = [np.arange(int(np.ceil(lo[a] - 1.5)), int(np.floor(hi[a] + 0.5)) + 1) for a in range(3)]
        X, Y, Z = np.meshgrid(*rng, indexing="ij")
        ck = (X.ravel() * (1 << 21) + Y.ravel()) * (1 << 21) + Z.ravel()
        pos = np.searchsorted(ks, ck)
        pos = np.minimum(pos, max(ks.size - 1, 0))
        hit = ks[pos] == ck if ks.size else np.zeros(ck.size, bool)
        idx = order[pos[hit]]
        if idx.size == 0:
            continue
        d = link_hits(tri, x[idx] + 0.5, y[idx] + 0.5, z[idx] + 0.5, q)
        cur = rows[idx]
        better = (d != -1.0) & ((cur == -1.0) | (d < cur))
        rows[idx] = np.where(better, d, cur)
    has = np.any(rows != -1.0, axis=1)
    return fluid_keys[has].copy(), rows[has].copy()


def _coords_of(keys, L, l):
    from .lattice import cell_coords
    return cell_coords(L, l, keys)


def _sphere_links(spec: MeshSpec, fluid_keys: np.ndarray):
    """Normalised distance from each finest-level fluid cell centre to the
    sphere along every link (Lat_Voxelize.cpp:1252-1285 semantics: 0 at the
    cell centre, 1 at the neighbour centre, -1 when the link is free)."""
    L = spec.max_level
    q = spec.q
    ex, ey, ez, _ = directions(q)
    s = 1 << L
    cx, cy, cz = (c * s for c in spec.sphere.center)
    r = spec.sphere.radius * s
    x, y, z = _coords_of(fluid_keys, L, L)
    px, py, pz = x + 0.5 - cx, y + 0.5 - cy, z + 0.5 - cz
    c0 = px * px + py * py + pz * pz - r * r
    rows = np.full((x.size, q - 1), -1.0)
    for d in range(1, q):
        a = float(ex[d] ** 2 + ey[d] ** 2 + ez[d] ** 2)
        b = 2.0 * (px * ex[d] + py * ey[d] + pz * ez[d])
        disc = b * b - 4.0 * a * c0
        ok = disc >= 0.0
        t = np.full(x.size, -1.0)
        t[ok] = (-b[ok] - np.sqrt(disc[ok])) / (2.0 * a)
        hit = ok & (t >= 0.0) & (t <= 1.0)
        rows[hit, d - 1] = t[hit]
    has = np.any(rows != -1.0, axis=1)
    return fluid_keys[has].copy(), rows[has].copy()


def cavity_or_box_spec(q, coarse, max_level=0, refine=None, boundary=("bc", "bc", "bc"), sphere=None):
    return MeshSpec(q=q, max_level=max_level, coarse=tuple(coarse), refine=list(refine or []),
                    boundary=tuple(boundary), sphere=sphere)
