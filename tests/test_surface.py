"""Triangulated solid surfaces (STL) on the host mesher: reading and writing
STL, the centre-inside classification and the link wall distances against
the analytic sphere and box they approximate, and the contract every solid
boundary must meet (a fluid link into the solid has a wall distance)."""
import numpy as np
import pytest


def _spec(surface=None, sphere=None, q=19):
    from mortontrie_amr_b200.mesh import MeshSpec
    return MeshSpec(q=q, max_level=1, coarse=(32, 16, 16), refine=[((6, 4, 4), (18, 12, 12))],
                    boundary=("bc", "periodic", "periodic"), surface=surface, sphere=sphere)


def test_stl_round_trip_ascii_and_binary(tmp_path):
    import struct
    from mortontrie_amr_b200.stl import icosphere, read_stl, write_stl
    tris = icosphere((1.0, 2.0, 3.0), 1.5, 1)
    write_stl(tmp_path / "a.stl", tris)
    got, normals = read_stl(tmp_path / "a.stl")
    assert np.array_equal(got, tris)
    # outward normals: the centre lies behind every facet
    assert np.all(np.einsum("ij,ij->i", normals, tris[:, 0] - np.array([1.0, 2.0, 3.0])) > 0)
    with open(tmp_path / "b.stl", "wb") as f:
        f.write(b"\0" * 80 + struct.pack("<I", len(tris)))
        for t, n in zip(tris.astype(np.float32), normals.astype(np.float32)):
            f.write(n.tobytes() + t.tobytes() + b"\0\0")
    got_b, _ = read_stl(tmp_path / "b.stl")
    assert np.array_equal(got_b, tris.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("sub", [2, 3])
def test_icosphere_matches_analytic_sphere(sub):
    from mortontrie_amr_b200.mesh import Sphere, build_mesh
    from mortontrie_amr_b200.stl import icosphere
    a = build_mesh(_spec(surface=icosphere((12, 8, 8), 2.0, sub)))
    b = build_mesh(_spec(sphere=Sphere((12, 8, 8), 2.0)))
    assert np.array_equal(a.levels[1]["lat_sf"], b.levels[1]["lat_sf"])
    assert np.array_equal(a.dis_keys, b.dis_keys)
    hit_a, hit_b = a.dis_rows != -1.0, b.dis_rows != -1.0
    assert np.array_equal(hit_a, hit_b)
    # the polyhedron lies inside the sphere: its walls are farther from the fluid
    err = np.abs(a.dis_rows[hit_a] - b.dis_rows[hit_b]).max()
    assert err < {2: 0.25, 3: 0.08}[sub]


def test_box_surface_exact():
    """An axis-aligned box: solid cells are exactly those with centres inside,
    and a link crossing a face has the exact normalised distance."""
    from mortontrie_amr_b200.lattice import cell_coords, directions
    from mortontrie_amr_b200.mesh import build_mesh
    from mortontrie_amr_b200.stl import box_surface
    lo, hi = np.array([10.3, 6.6, 6.1]), np.array([13.7, 9.4, 9.85])
    m = build_mesh(_spec(surface=box_surface(lo, hi)))
    x, y, z = cell_coords(1, 1, m.levels[1]["lat_sf"])
    c = np.stack([x, y, z]) + 0.5
    assert np.all((c > 2 * lo[:, None]) & (c < 2 * hi[:, None]))
    n = np.prod([np.sum((np.arange(64) + 0.5 > 2 * lo[a]) & (np.arange(64) + 0.5 < 2 * hi[a])) for a in range(3)])
    assert x.size == n
    ex, ey, ez, _ = directions(19)
    kx, ky, kz = cell_coords(1, 1, m.dis_keys)
    for j in range(m.dis_keys.size):
        p = np.array([kx[j], ky[j], kz[j]]) + 0.5
        for k in range(1, 19):
            e = np.array([ex[k], ey[k], ez[k]], float)
            ts = []
            for a in range(3):
                for w in (2 * lo[a], 2 * hi[a]):
                    if e[a] != 0:
                        t = (w - p[a]) / e[a]
                        pt = p + t * e
                        inside = all(2 * lo[b] - 1e-12 <= pt[b] <= 2 * hi[b] + 1e-12 for b in range(3) if b != a)
                        if 0 < t <= 1 and inside:
                            ts.append(t)
            want = min(ts) if ts else -1.0
            assert abs(m.dis_rows[j, k - 1] - want) < 1e-12, (j, k, m.dis_rows[j, k - 1], want)


@pytest.mark.parametrize("q", [19, 27])
def test_fluid_links_into_the_solid_have_a_wall(q):
    from mortontrie_amr_b200.lattice import cell_coords, cell_key, directions
    from mortontrie_amr_b200.mesh import build_mesh
    from mortontrie_amr_b200.stl import box_surface, icosphere
    for surf in (icosphere((12, 8, 8), 2.3, 2), box_surface((10.3, 6.6, 6.1), (13.7, 9.4, 9.85))):
        m = build_mesh(_spec(surface=surf, q=q))
        solid = set(m.levels[1]["lat_sf"].tolist())
        rows = dict(zip(m.dis_keys.tolist(), m.dis_rows))
        ex, ey, ez, _ = directions(q)
        x, y, z = cell_coords(1, 1, m.levels[1]["lat_f"])
        for k in range(1, q):
            nk = cell_key(1, 1, x + ex[k], y + ey[k], z + ez[k])
            into = np.array([v in solid for v in nk.tolist()])
            for key in m.levels[1]["lat_f"][into].tolist():
                assert key in rows and rows[key][k - 1] != -1.0, (key, k)


def _min_barycentric(tri, p, k, q):
    """Smallest barycentric coordinate of link k's crossing of one triangle
    (Moller-Trumbore, as Shape::intersect_line_with_triangle), None if the
    link runs parallel to it or the crossing lies behind the centre."""
    from mortontrie_amr_b200.lattice import directions
    ex, ey, ez, _ = directions(q)
    d = np.array([ex[k], ey[k], ez[k]], float)
    d /= np.linalg.norm(d)
    e1, e2, s = tri[1] - tri[0], tri[2] - tri[0], p - tri[0]
    s1 = np.cross(d, e2)
    den = s1 @ e1
    if den == 0.0:
        return None
    s2 = np.cross(s, e1)
    t, b1, b2 = (s2 @ e2) / den, (s1 @ s) / den, (s2 @ d) / den
    return min(b1, b2, 1.0 - b1 - b2) if t > 0 else None


@pytest.mark.parametrize("name", ["dis_icosphere_q19", "dis_icosphere_q27"])
def test_links_match_reference_compute_distance(name):
    """The mesher's link wall distances against the distances the reference's
    own Lat_Manager::compute_distance (Lat_Voxelize.cpp:1252-1285, through
    Shape::intersect_line_with_triangle, Shape.cpp:809-843) gave for the same
    triangles and cell centres (golden, made by the reference harness).
    Bit-exact on every link both define.  The reference drops a crossing whose
    barycentric coordinates are not all >= 1e-10, i.e. one on a triangle's
    edge or vertex; the mesher keeps those (>= -1e-10) so that a link through
    an edge shared by two triangles is not missed, and that is the only
    difference allowed."""
    import json
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from golden_cases import dis_mesh
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    spec = json.loads(bytes(g["meta"]).decode())
    q = spec["q"]
    mesh, tris = dis_mesh(spec)
    keys, ref = g["keys"], g["dis"]
    ours = np.full_like(ref, -1.0)
    pos = np.minimum(np.searchsorted(mesh.dis_keys, keys), mesh.dis_keys.size - 1)
    has = mesh.dis_keys[pos] == keys
    ours[has] = mesh.dis_rows[pos[has]]
    both = (ref != -1.0) & (ours != -1.0)
    assert both.sum() > 1000
    assert np.array_equal(ref[both], ours[both])
    assert not np.any((ref != -1.0) & (ours == -1.0))
    from mortontrie_amr_b200.lattice import cell_coords
    for i, j in zip(*np.nonzero((ours != -1.0) & (ref == -1.0))):
        x, y, z = cell_coords(1, 1, keys[i:i + 1])
        p = (np.array([x[0], y[0], z[0]], float) + 0.5) / 2.0
        bs = [b for b in (_min_barycentric(t, p, j + 1, q) for t in tris) if b is not None and abs(b) < 1e-9]
        assert bs and min(abs(b) for b in bs) < 1e-10
