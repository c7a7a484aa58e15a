"""Flow output in the reference's Tecplot format: the vectorised writer
against a loop-by-loop restatement of IO_TECPLOTH::write (tecplot.cpp:16-176)
on small multi-level meshes, and the file's structure."""
import numpy as np
import pytest


def _levels(case, seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for l in range(case.max_level + 1):
        keys = np.concatenate([case.mesh.levels[l]["lat_f"], case.mesh.levels[l]["overlap_F2C"]])
        out.append((keys, rng.uniform(-0.1, 0.1, (3, keys.size))))
    return out


def _loops(levels, L):
    """tecplot.cpp:27-79 and 146-171 as written: a dict of first-seen nodes."""
    from mortontrie_amr_b200.lattice import cell_coords, cell_key

    def step(key, l, dx, dy, dz):
        x, y, z = (int(v[0]) for v in cell_coords(L, l, np.array([key], np.uint64)))
        return int(cell_key(L, l, np.array([x + dx]), np.array([y + dy]), np.array([z + dz]))[0])

    node, order = {}, []
    for l, (keys, _) in enumerate(levels):
        for k in keys.tolist():
            for o in [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1)]:
                v = step(k, l, *o)
                if v not in node:
                    node[v] = (len(node) + 1, l)
                    order.append(v)
    conn = []
    for l, (keys, _) in enumerate(levels):
        for k in keys.tolist():
            conn.append([node[step(k, l, *o)][0] for o in [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1),
                                                            (1, 0, 1), (1, 1, 1), (0, 1, 1)]])
    return order, [node[v][1] for v in order], conn


def _coord_loop(key, level, L, dx, axis):
    """Morton_Assist::compute_coordinate (3-D form) bit by bit."""
    v = 0.0
    for i in range(1, level + 1):
        if (key >> (3 * (L - i) + axis)) & 1:
            v += dx / 2 ** i
    for i in range(0, 21 - L):
        if (key >> (3 * (L + i) + axis)) & 1:
            v += dx * 2 ** i
    return v


@pytest.mark.parametrize("which", ["cavity_l1", "sphere_l2"])
def test_zone_matches_reference_loops(which):
    from mortontrie_amr_b200.case import cavity_case, nested_sphere_case
    from mortontrie_amr_b200.tecplot import flow_zone, node_coordinates
    case = (cavity_case(coarse=(8, 8, 8), max_level=1, refine=[((2, 2, 4), (6, 6, 7))]) if which == "cavity_l1" else
            nested_sphere_case(coarse=(24, 12, 12), max_level=2, center=(8, 6, 6), radius=1.0,
                               half_widths=(4.0, 2.5)))
    L = case.max_level
    levels = _levels(case)
    keys, lev, conn, u = flow_zone(levels, L)
    order, olev, oconn = _loops(levels, L)
    assert keys.tolist() == order
    assert lev.tolist() == olev
    assert conn.tolist() == oconn
    assert np.array_equal(u, np.concatenate([uv for _, uv in levels], axis=1))
    dx = 0.37
    xyz = node_coordinates(keys, lev, L, dx)
    for a in range(3):
        want = [_coord_loop(k, l, L, dx, a) for k, l in zip(order, olev)]
        assert xyz[a].tolist() == want


def test_file_structure(tmp_path):
    from mortontrie_amr_b200.case import cavity_case
    from mortontrie_amr_b200.tecplot import flow_zone, write_zone
    case = cavity_case(coarse=(8, 8, 8), max_level=1, refine=[((2, 2, 4), (6, 6, 7))])
    levels = _levels(case)
    keys, lev, conn, u = flow_zone(levels, 1)
    path = tmp_path / "sphereFlow_1.000000.dat"
    write_zone(str(path), keys, lev, conn, u, 1, dx=1.0, u_scale=2.0)
    lines = path.read_text().splitlines()
    assert lines[0] == 'TITLE = "Flow Field Example"'
    assert lines[1] == 'VARIABLES = "X", "Y", "Z", "U", "V", "W"'
    n, e = keys.size, conn.shape[0]
    assert lines[2] == (f"ZONE, NODES={n}, ELEMENTS={e}, DATAPACKING=BLOCK, VARLOCATION=([4,5,6]=CELLCENTERED), "
                        "ZONETYPE=FEBRICK")
    body = lines[3:]
    assert len(body) == 3 * n + 3 * e + e
    xyz = np.array([float(v) for v in body[:3 * n]]).reshape(3, n)
    uu = np.array([float(v) for v in body[3 * n:3 * n + 3 * e]]).reshape(3, e)
    assert np.allclose(uu, 2.0 * u, rtol=1e-5, atol=1e-7)
    cells = np.array([[int(t) for t in r.split()] for r in body[3 * n + 3 * e:]]) - 1
    # every element is an axis-aligned cube of its level's size, corners in FEBRICK order
    size = np.concatenate([np.full(k.size, 1.0 / (1 << l)) for l, (k, _) in enumerate(levels)])
    p = xyz[:, cells]                                 # [3][e][8]
    d = p - p[:, :, :1]
    want = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]).T
    assert np.allclose(d, want[:, None, :] * size[None, :, None])
    # no two nodes at the same point
    assert np.unique(xyz.T, axis=0).shape[0] == n
