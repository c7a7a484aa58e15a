"""Refinement made from the body (an octree of 2:1-nested levels) instead of
boxes: the region operations against brute force, the box regions through
the same code path against the box mesher, and the invariants of the
index-set contract (Lat_Manager.hpp:245-316) on octree meshes of spheres
and STL surfaces."""
import numpy as np
import pytest

from mortontrie_amr_b200.lattice import cell_coords, cell_key
from mortontrie_amr_b200.mesh import MeshSpec, Octree, Region, Sphere, box_region, build_mesh


def _grid_around(lo, hi, pad):
    g = np.meshgrid(*[np.arange(a - pad, b + pad) for a, b in zip(lo, hi)], indexing="ij")
    return [v.ravel() for v in g]


def test_region_operations_match_brute_force():
    rng = np.random.default_rng(0)
    r = Region((1, -2, 3), rng.random((7, 6, 5)) < 0.1)
    xs, ys, zs = r.cells()
    gx, gy, gz = _grid_around(r.lo, r.hi, 4)
    near = np.zeros(gx.size, bool)
    for a, b, c in zip(xs, ys, zs):
        near |= (np.abs(gx - a) <= 2) & (np.abs(gy - b) <= 2) & (np.abs(gz - c) <= 2)
    assert np.array_equal(near, r.dilate(2).contains(gx, gy, gz))
    allin = np.ones(gx.size, bool)
    for d in np.ndindex(3, 3, 3):
        allin &= r.contains(gx + d[0] - 1, gy + d[1] - 1, gz + d[2] - 1)
    assert np.array_equal(r.contains(gx, gy, gz) & ~allin, r.shell().contains(gx, gy, gz))
    par = np.zeros(gx.size, bool)
    for a, b, c in zip(xs, ys, zs):
        par |= (gx == a // 2) & (gy == b // 2) & (gz == c // 2)
    p = r.parents()
    assert np.array_equal(par, p.contains(gx, gy, gz))
    assert np.array_equal(p.contains(gx // 2, gy // 2, gz // 2), p.children().contains(gx, gy, gz))


def _box_specs():
    from mortontrie_amr_b200.stl import icosphere
    yield MeshSpec(q=19, max_level=1, coarse=(32, 16, 16), refine=[((6, 4, 4), (18, 12, 12))],
                   boundary=("bc", "periodic", "periodic"), sphere=Sphere((12, 8, 8), 2.0))
    from mortontrie_amr_b200.case import nested_sphere_case
    yield nested_sphere_case(coarse=(48, 24, 24), center=(16, 12, 12), radius=1.5).mesh.spec
    yield MeshSpec(q=19, max_level=2, coarse=(32, 16, 16), refine=[((6, 3, 3), (20, 13, 13)), ((16, 10, 10), (36, 22, 22))],
                   boundary=("bc", "bc", "bc"), surface=icosphere((12.3, 8.1, 7.9), 2.2, 2))


def _same_mesh(a, b):
    assert len(a.levels) == len(b.levels)
    for la, lb in zip(a.levels, b.levels):
        assert sorted(la) == sorted(lb)
        for k in la:
            assert np.array_equal(la[k], lb[k]), k
    for x, y in zip(a.lat_bc, b.lat_bc):
        assert np.array_equal(x, y)
    assert np.array_equal(a.dis_keys, b.dis_keys) and np.array_equal(a.dis_rows, b.dis_rows)


@pytest.mark.parametrize("which", [0, 1, 2])
def test_box_regions_reproduce_the_box_mesher(monkeypatch, which):
    """The octree code path fed the boxes as regions gives the box mesher's
    sets exactly: F2C = the region's outer layer, C2F = its children."""
    import dataclasses
    import mortontrie_amr_b200.mesh as M
    spec = list(_box_specs())[which]
    want = build_mesh(spec)
    regions = [None] + [box_region(lo, hi) for lo, hi in spec.refine]
    monkeypatch.setattr(M, "octree_regions", lambda s: regions)
    got = build_mesh(dataclasses.replace(spec, refine=[], octree=Octree()))
    _same_mesh(want, got)


def _octree_specs():
    from mortontrie_amr_b200.stl import icosphere
    for L in (1, 2, 3):
        yield f"sphere_l{L}", MeshSpec(q=19, max_level=L, coarse=(48, 24, 24), boundary=("bc", "periodic", "periodic"),
                                       sphere=Sphere((16.0, 12.0, 12.0), 2.5), octree=Octree())
    yield "stl_q27_l2", MeshSpec(q=27, max_level=2, coarse=(48, 24, 24), boundary=("bc", "bc", "bc"),
                                 surface=icosphere((16.3, 12.1, 11.8), 2.5, 3), octree=Octree(band=2.0, margin=5))


@pytest.mark.parametrize("name,spec", list(_octree_specs()), ids=[n for n, _ in _octree_specs()])
def test_octree_mesh_contract(name, spec):
    """Sets disjoint; C2F[l] = the children of F2C[l-1], all stored; the
    leaves (lat_f, C2F, solid and the boundary shell of every level) tile the
    domain exactly once; the finest level holds the body and its band."""
    m = build_mesh(spec)
    L = spec.max_level
    names = ["lat_f", "overlap_F2C", "overlap_C2F", "ghost_overlap_C2F", "lat_sf"]
    for l in range(L + 1):
        s = m.levels[l]
        for i, a in enumerate(names):
            for b in names[i + 1:]:
                assert not np.intersect1d(s[a], s[b]).size, (l, a, b)
        assert np.all(np.isin(s["ghost_overlap_F2C"], s["lat_f"]))
        if l > 0:
            x, y, z = cell_coords(L, l - 1, m.levels[l - 1]["overlap_F2C"])
            kids = np.unique(np.concatenate([cell_key(L, l, 2 * x + d[0], 2 * y + d[1], 2 * z + d[2])
                                             for d in np.ndindex(2, 2, 2)]))
            assert np.array_equal(kids, s["overlap_C2F"]), l
            assert np.all(np.isin(kids, m.all_keys(l)))
    # tiling: every finest-level cell of the domain under exactly one leaf
    ext = np.array(spec.coarse) << L
    count = np.zeros(tuple(ext.tolist()), np.int32)
    bc = np.concatenate(m.lat_bc)
    for l in range(L + 1):
        s = m.levels[l]
        leaves = np.concatenate([s["lat_f"], s["overlap_C2F"], s["lat_sf"]] + ([bc] if l == 0 else []))
        x, y, z = cell_coords(L, l, leaves)
        w = 1 << (L - l)
        for d in np.ndindex(w, w, w):
            np.add.at(count, (w * x + d[0], w * y + d[1], w * z + d[2]), 1)
    assert count.min() == 1 and count.max() == 1
    # the body and every cell within the band of its surface are on the finest level
    fine = m.all_keys(L)
    x, y, z = cell_coords(L, L, fine)
    s = 1 << L
    if spec.sphere is not None:
        c, r = np.array(spec.sphere.center) * s, spec.sphere.radius * s
        g = np.stack(np.meshgrid(*[np.arange(int(c[a] - r) - 8, int(c[a] + r) + 8) for a in range(3)],
                                 indexing="ij")).reshape(3, -1)
        d = np.linalg.norm(g + 0.5 - c[:, None], axis=0)
        need = g[:, d <= r + spec.octree.band * 2 ** (L - (L - 1)) - 1.0]
        have = set(zip(x.tolist(), y.tolist(), z.tolist()))
        assert all(tuple(v) in have for v in need.T.tolist())
    assert m.levels[L]["lat_sf"].size > 0 and m.dis_keys.size > 0


def _tiles_once(m):
    L = m.spec.max_level
    ext = np.array(m.spec.coarse) << L
    count = np.zeros(tuple(ext.tolist()), np.int32)
    bc = np.concatenate(m.lat_bc)
    for l in range(L + 1):
        s = m.levels[l]
        leaves = np.concatenate([s["lat_f"], s["overlap_C2F"], s["lat_sf"]] + ([bc] if l == 0 else []))
        x, y, z = cell_coords(L, l, leaves)
        w = 1 << (L - l)
        for d in np.ndindex(w, w, w):
            np.add.at(count, (w * x + d[0], w * y + d[1], w * z + d[2]), 1)
    return count.min() == 1 and count.max() == 1


@pytest.mark.parametrize("osc", [False, True])
def test_octree_direct_forcing_sphere(osc):
    """A direct-forcing sphere refined around its forcing band and path: the
    same band as the boxes give, the fluid inside on coarser levels, every
    C2F cell a child of an F2C cell, the leaves tiling the domain once."""
    from mortontrie_amr_b200.case import df_sphere_case
    oc = df_sphere_case(radius=3, max_level=2, oscillating=osc, octree=Octree(band=2.0, margin=4)).mesh
    box = df_sphere_case(radius=3, max_level=2, oscillating=osc).mesh
    L = 2
    assert np.array_equal(oc.levels[L]["ib_band"], box.levels[L]["ib_band"])
    assert oc.n_cells()[L] < box.n_cells()[L]
    for l in range(1, L + 1):
        x, y, z = cell_coords(L, l - 1, oc.levels[l - 1]["overlap_F2C"])
        kids = np.unique(np.concatenate([cell_key(L, l, 2 * x + d[0], 2 * y + d[1], 2 * z + d[2])
                                         for d in np.ndindex(2, 2, 2)]))
        assert np.array_equal(kids, oc.levels[l]["overlap_C2F"]), l
    assert _tiles_once(oc)
    if not osc:
        # the sphere's centre is not on the finest level (hollow region; a
        # path of amplitude R/2 sweeps the band over the centre of so small a sphere)
        s = 1 << L
        c = [int(v * s) for v in oc.spec.sphere.center]
        fine = set(zip(*[v.tolist() for v in cell_coords(L, L, oc.all_keys(L))]))
        assert tuple(c) not in fine
    assert np.array_equal(oc.markers.ref, box.markers.ref) and np.array_equal(oc.markers.path, box.markers.path)


def test_octree_smaller_than_boxes():
    """The 4-level sphere: the octree's finest level covers the body and its
    band, far fewer cells than the nested box of the same sphere."""
    from mortontrie_amr_b200.case import nested_sphere_case
    from mortontrie_amr_b200.mesh import estimate_cells
    box = nested_sphere_case(coarse=(96, 48, 48), center=(32, 24, 24), radius=3.0).mesh
    spec = MeshSpec(q=27, max_level=3, coarse=(96, 48, 48), boundary=("bc", "periodic", "periodic"),
                    sphere=Sphere((32.0, 24.0, 24.0), 3.0), octree=Octree(band=3.0, margin=4))
    oc = build_mesh(spec)
    assert oc.n_cells()[3] < box.n_cells()[3] / 2
    est = estimate_cells(spec)
    assert all(e >= n for e, n in zip(est, oc.n_cells()))


def test_octree_errors():
    from mortontrie_amr_b200.mesh import spec_mesh
    base = dict(q=19, max_level=2, coarse=(32, 16, 16), boundary=("bc", "periodic", "periodic"))
    with pytest.raises(ValueError, match="exclusive"):
        build_mesh(MeshSpec(refine=[((4, 4, 4), (12, 12, 12))] * 2, sphere=Sphere((8, 8, 8), 1.0), octree=Octree(),
                            **base))
    with pytest.raises(ValueError, match="leaves the domain"):
        build_mesh(MeshSpec(sphere=Sphere((3.0, 8.0, 8.0), 1.5), octree=Octree(), **base))
    with pytest.raises(ValueError, match="made from a body"):
        build_mesh(MeshSpec(octree=Octree(), **base))
    with pytest.raises(ValueError, match="leaves the domain"):
        spec_mesh(MeshSpec(sphere=Sphere((3.0, 8.0, 8.0), 1.5), octree=Octree(), **base))
    ok = spec_mesh(MeshSpec(sphere=Sphere((16.0, 8.0, 8.0), 1.5), octree=Octree(), **base))
    assert ok.spec.octree is not None


def _octree_cases():
    from mortontrie_amr_b200.case import sphere_case, surface_case
    from mortontrie_amr_b200.stl import icosphere
    return {
        "sphere_q19_l2": lambda: sphere_case(coarse=(48, 24, 24), max_level=2, center=(16, 12, 12), radius=2.5,
                                             octree=Octree()),
        "stl_q27_l2": lambda: surface_case(icosphere((16.3, 12.1, 11.8), 2.5, 3), q=27, collision="Cumulant",
                                           coarse=(48, 24, 24), max_level=2, octree=Octree(band=2.0, margin=5)),
    }


@pytest.mark.parametrize("which", ["sphere_q19_l2", "stl_q27_l2"])
def test_octree_case_steps_on_the_oracle(which):
    """An octree case runs through the oracle's multi-level step (the sets
    satisfy its contract checks) and stays finite with a drag on the body."""
    from helpers import run_oracle
    case = _octree_cases()[which]()
    oc = run_oracle(case, 3)
    for l in range(case.max_level + 1):
        assert np.isfinite(oc.get(l)["f"]).all(), l
    assert oc.force()[3] > 0 and np.isfinite(oc.force()[:3]).all()
