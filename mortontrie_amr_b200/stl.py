"""Triangulated solid surfaces (STL) for the lattice classification.

The reference reads ASCII STL in Shape::geofile_stl (Shape.cpp:341-470):
"facet normal nx ny nz / outer loop / vertex x y z (x3) / endloop /
endfacet".  read_stl accepts that form and binary STL; the triangles are
returned as an (n, 3, 3) float64 array (vertex, axis), with the facet normals
(n, 3).  icosphere and box_surface make closed test surfaces with outward
normals and counter-clockwise vertices.
"""
from __future__ import annotations

import struct

import numpy as np


def read_stl(path):
    """(triangles (n,3,3), normals (n,3)) of an ASCII or binary STL file."""
    with open(path, "rb") as f:
        data = f.read()
    if len(data) >= 84:
        n = struct.unpack("<I", data[80:84])[0]
        if len(data) == 84 + 50 * n:
            rec = np.frombuffer(data, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]),
                                count=n, offset=84)
            return rec["v"].astype(np.float64), rec["n"].astype(np.float64)
    tris, norms, cur = [], [], []
    for raw in data.decode("ascii", errors="replace").splitlines():
        tok = raw.split()
        if not tok:
            continue
        if tok[0] == "facet":
            if len(tok) < 5 or tok[1] != "normal":
                raise ValueError(f"expected 'facet normal', got {raw.strip()!r}")
            norms.append([float(t) for t in tok[2:5]])
            cur = []
        elif tok[0] == "vertex":
            cur.append([float(t) for t in tok[1:4]])
        elif tok[0] == "endfacet":
            if len(cur) != 3:
                raise ValueError("a facet without three vertices")
            tris.append(cur)
    if not tris:
        raise ValueError(f"no facets in {path}")
    return np.array(tris, np.float64), np.array(norms, np.float64)


def write_stl(path, tris, name="solid"):
    """ASCII STL with normals from the vertex order."""
    tris = np.asarray(tris, np.float64)
    n = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-300)
    with open(path, "w") as f:
        f.write(f"solid {name}\n")
        for t, nn in zip(tris, n):
            f.write(f"  facet normal {nn[0]:.9e} {nn[1]:.9e} {nn[2]:.9e}\n    outer loop\n")
            for v in t:
                f.write(f"      vertex {v[0]:.17g} {v[1]:.17g} {v[2]:.17g}\n")
            f.write("    endloop\n  endfacet\n")
        f.write(f"endsolid {name}\n")


def icosphere(center, radius, subdivisions=3):
    """Closed triangulated sphere: an icosahedron refined `subdivisions`
    times, vertices projected onto the sphere (20 * 4^s triangles)."""
    p = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
         (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.array(x, np.float64) / np.linalg.norm(x) for x in v]
    for _ in range(subdivisions):
        mid = {}

        def m(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                c = verts[a] + verts[b]
                verts.append(c / np.linalg.norm(c))
                mid[k] = len(verts) - 1
            return mid[k]
        nf = []
        for a, b, c in f:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    V = np.array(verts) * float(radius) + np.asarray(center, np.float64)
    return V[np.array(f)]


def box_surface(lo, hi):
    """Closed axis-aligned box [lo, hi] as 12 triangles, outward normals."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    c = np.array([(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0),
                  (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)], np.float64)
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (2, 3, 7, 6), (1, 2, 6, 5), (0, 4, 7, 3)]
    tris = []
    for a, b, cc, d in quads:
        tris += [(a, b, cc), (a, cc, d)]
    return c[np.array(tris)]
