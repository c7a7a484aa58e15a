"""Flow output in the reference's Tecplot format: the vectorised writer
against a loop-by-loop restatement of IO_TECPLOTH::write (tecplot.cpp:16-176)
on small multi-level meshes, the file's structure, and the file the
reference's own IO_TECPLOTH::write produced (golden)."""
import os

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


def _parse_flow(text):
    """(nodes, elements) of a FEBRICK flow file: elements keyed by the
    coordinate strings of their 8 corners in connectivity order, with their
    U, V, W strings."""
    lines = text.splitlines()
    head = lines[2]
    nn = int(head.split("NODES=")[1].split(",")[0])
    ne = int(head.split("ELEMENTS=")[1].split(",")[0])
    body = lines[3:]
    x, y, z = body[:nn], body[nn:2 * nn], body[2 * nn:3 * nn]
    u = body[3 * nn:3 * nn + ne]
    v = body[3 * nn + ne:3 * nn + 2 * ne]
    w = body[3 * nn + 2 * ne:3 * nn + 3 * ne]
    conn = body[3 * nn + 3 * ne:]
    assert len(conn) == ne
    nodes = [(x[i], y[i], z[i]) for i in range(nn)]
    elems = {}
    for j, row in enumerate(conn):
        corners = tuple(nodes[int(t) - 1] for t in row.split())
        assert corners not in elems
        elems[corners] = (u[j], v[j], w[j])
    return lines[:3], nodes, elems


def test_flow_file_matches_reference_output():
    """write_flow against the file the reference's own IO_TECPLOTH::write
    produced (tests/golden/tecplot_sphere_q19_fh_refinit.npz, 3 coarse steps
    of the 2-level FH sphere, iteration 7): same header and counts, the same
    set of node coordinates, and every element -- its 8 corner coordinates in
    connectivity order -- with the same velocity text.  The reference built
    with hash maps visits cells in hash order, so nodes and elements are
    compared as sets, not by position."""
    import json

    from golden_cases import build_case
    from helpers import GOLDEN_DIR, run_oracle
    from mortontrie_amr_b200.tecplot import write_flow
    z = np.load(os.path.join(GOLDEN_DIR, "tecplot_sphere_q19_fh_refinit.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    ref_text = bytes(z["text"]).decode()
    from golden_cases import GOLDEN_CASES
    case = build_case(GOLDEN_CASES[meta["case"]])
    oc = run_oracle(case, meta["steps"])

    class View:
        L = case.max_level

        def keys(self, l):
            g = oc.get(l)
            return g["keys"], g["tags"]

        def macros(self, l):
            g = oc.get(l)
            return g["rho"], np.ascontiguousarray(g["u"].T)

    import tempfile
    with tempfile.TemporaryDirectory() as td:
        path = write_flow(View(), td, meta["iteration"])
        assert os.path.basename(path) == meta["file"]
        with open(path) as fh:
            ours = fh.read()
    h1, n1, e1 = _parse_flow(ours)
    h0, n0, e0 = _parse_flow(ref_text)
    assert h1 == h0
    assert sorted(n1) == sorted(n0)
    assert e1 == e0
