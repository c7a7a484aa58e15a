"""Flow output in the reference's Tecplot format (IO_TECPLOTH::write,
tecplot.cpp:16-176).

One ASCII FEBRICK zone over the cells of every level: for each level, its
lat_f cells then its overlap_F2C cells (ascending Morton order, the order the
reference's MortonTrie maps iterate in).  Nodes are the cells' corner keys,
numbered from 1 in order of first appearance, with each cell's corners
visited as (0,0,0), x+1, y+1, z+1, x+1 y+1, x+1 z+1, y+1 z+1, x+1 y+1 z+1 at
the cell's level (tecplot.cpp:33-78); a corner is the key of the same-level
cell one step further, so coincident corners of different levels share a
node.  Then X, Y, Z of every node (Morton_Assist::compute_coordinate,
Morton_Assist.cpp:203-238, the three-dimensional form: 0, plus dx / 2^i for
each set bit of refinement level i = 1..l, plus dx 2^i for each set bit of
the background key, summed in that order; `origin` shifts it), U, V, W of
every cell (cell-centred, times the velocity conversion factor), and the
connectivity in the order (0,0,0),
x+1, x+1 y+1, y+1, z+1, x+1 z+1, x+1 y+1 z+1, y+1 z+1 (tecplot.cpp:146-171).
Numbers are written as C++ streams write doubles by default (%g, six
significant digits).
"""
from __future__ import annotations

import os

import numpy as np

from .lattice import _compact3, _dilate3

TAG_LATF = 1
TAG_F2C = 2

# corner offsets in node-numbering order and in connectivity order
_VISIT = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1)]
_CONN = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]


def _corner_keys(keys, L, level, off):
    """Keys of the same-level cells at +off (the reference's find_x1 / find_y1
    / find_z1 compositions: masked increments, no wrap)."""
    sh = np.uint64(L - level)
    out = np.zeros(keys.size, np.uint64)
    for a in range(3):
        c = (_compact3(keys >> np.uint64(a)) >> sh) + np.uint64(off[a])
        out |= _dilate3(c << sh) << np.uint64(a)
    return out


def node_coordinates(node_keys, node_level, L, dx=1.0, origin=(0.0, 0.0, 0.0)):
    """compute_coordinate of each node at the level it was first seen on."""
    xyz = []
    for a in range(3):
        v = np.full(node_keys.size, float(origin[a]))
        c = _compact3(node_keys >> np.uint64(a))
        for i in range(1, L + 1):
            bit = ((c >> np.uint64(L - i)) & np.uint64(1)).astype(bool) & (node_level >= i)
            v[bit] += dx / float(1 << i)
        for i in range(0, 21 - L):
            bit = ((c >> np.uint64(L + i)) & np.uint64(1)).astype(bool)
            v[bit] += dx * float(1 << i)
        xyz.append(v)
    return xyz


def flow_zone(levels, L):
    """levels[l] = (keys, u): the level's written cells in order (lat_f then
    F2C) and their velocity [3][n].  Returns (node_keys, node_level,
    connectivity [n_cells][8] 1-based, u [3][n_cells])."""
    visit = []
    lev = []
    for l, (keys, _) in enumerate(levels):
        if keys.size == 0:
            continue
        corners = np.stack([_corner_keys(keys, L, l, o) for o in _VISIT], axis=1)  # [n][8]
        visit.append(corners.ravel())
        lev.append(np.full(corners.size, l, np.int64))
    if not visit:
        return np.zeros(0, np.uint64), np.zeros(0, np.int64), np.zeros((0, 8), np.int64), np.zeros((3, 0))
    visit = np.concatenate(visit)
    lev = np.concatenate(lev)
    uniq, first, inv = np.unique(visit, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")       # nodes in order of first appearance
    rank = np.empty(uniq.size, np.int64)
    rank[order] = np.arange(1, uniq.size + 1)
    node_keys = uniq[order]
    node_level = lev[first[order]]
    conn = []
    for l, (keys, _) in enumerate(levels):
        if keys.size == 0:
            continue
        c = np.stack([_corner_keys(keys, L, l, o) for o in _CONN], axis=1)
        conn.append(rank[np.searchsorted(uniq, c)])
    u = np.concatenate([np.asarray(uv, np.float64).reshape(3, -1) for _, uv in levels], axis=1)
    return node_keys, node_level, np.concatenate(conn), u


def _g(values) -> str:
    return "\n".join("%g" % v for v in values.tolist()) + ("\n" if values.size else "")


def write_zone(path, node_keys, node_level, conn, u, L, dx=1.0, origin=(0.0, 0.0, 0.0), u_scale=1.0):
    x, y, z = node_coordinates(node_keys, node_level, L, dx, origin)
    with open(path, "w") as f:
        f.write('TITLE = "Flow Field Example"\n')
        f.write('VARIABLES = "X", "Y", "Z", "U", "V", "W"\n')
        f.write(f"ZONE, NODES={node_keys.size}, ELEMENTS={conn.shape[0]}, DATAPACKING=BLOCK, "
                "VARLOCATION=([4,5,6]=CELLCENTERED), ZONETYPE=FEBRICK\n")
        for v in (x, y, z):
            f.write(_g(v))
        for a in range(3):
            f.write(_g(u[a] * u_scale))
        f.write("".join(" ".join(map(str, row)) + " \n" for row in conn.tolist()))


def write_flow(mgr, out_dir: str, iteration: int, dx: float = 1.0, origin=(0.0, 0.0, 0.0), u_scale: float = 1.0,
               t_scale: float = 1.0) -> str:
    """Write the case's current velocity field as
    out_dir/sphereFlow_<iteration * t_scale>.dat (IO_Manager::writeFlow).
    dx: level-0 cell size (C_dx); u_scale: velocity conversion (CF_U);
    t_scale: time per coarse step (CF_T[0])."""
    levels = []
    for l in range(mgr.L + 1):
        keys, tags = mgr.keys(l)
        _, u = mgr.macros(l)
        sel = np.concatenate([np.flatnonzero(tags & TAG_LATF), np.flatnonzero(tags & TAG_F2C)])
        levels.append((keys[sel], u[:, sel]))
    node_keys, node_level, conn, u = flow_zone(levels, mgr.L)
    path = os.path.join(out_dir, "sphereFlow_%f.dat" % (iteration * t_scale))
    write_zone(path, node_keys, node_level, conn, u, mgr.L, dx, origin, u_scale)
    return path
