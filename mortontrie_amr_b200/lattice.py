"""Lattice tables, Morton keys and unit conversion shared by the host side.

The direction ordering, weights and inverse table follow the reference's
D3Q19 / D3Q27 definitions (header/Constants.h:492-538 for ex/ey/ez/e_inv,
LBM_Manager.cpp:137-169 for the weights).  The Morton layout follows
Morton_Assist.cpp:20-106,185-193: x, y, z interleaved as bits 3k, 3k+1,
3k+2 of the finest-level coordinate, so a level-l cell at (x, y, z) has the
key morton(x << (L-l), y << (L-l), z << (L-l)) with L = the maximum level.
"""
from __future__ import annotations

import numpy as np

EX19 = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0], np.int64)
EY19 = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1], np.int64)
EZ19 = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1], np.int64)

EX27 = np.concatenate([EX19, np.array([1, -1, 1, -1, -1, 1, -1, 1], np.int64)])
EY27 = np.concatenate([EY19, np.array([1, -1, -1, 1, -1, 1, 1, -1], np.int64)])
EZ27 = np.concatenate([EZ19, np.array([1, -1, 1, -1, 1, -1, 1, -1], np.int64)])


def directions(q: int):
    """(ex, ey, ez, inv) for D3Q19 or D3Q27 in the reference ordering."""
    if q == 19:
        ex, ey, ez = EX19, EY19, EZ19
    elif q == 27:
        ex, ey, ez = EX27, EY27, EZ27
    else:
        raise ValueError(f"unsupported lattice Q={q}")
    inv = np.zeros(q, np.int64)
    for i in range(q):
        for j in range(q):
            if ex[j] == -ex[i] and ey[j] == -ey[i] and ez[j] == -ez[i]:
                inv[i] = j
    return ex, ey, ez, inv


def weights(q: int) -> np.ndarray:
    if q == 19:
        return np.array([1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12)
    if q == 27:
        return np.array([8.0 / 27.0] + [2.0 / 27.0] * 6 + [1.0 / 54.0] * 12 + [1.0 / 216.0] * 8)
    raise ValueError(f"unsupported lattice Q={q}")


def _dilate3(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint64) & np.uint64(0x1FFFFF)
    v = (v | (v << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    v = (v | (v << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    v = (v | (v << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    v = (v | (v << np.uint64(2))) & np.uint64(0x1249249249249249)
    return v


def _compact3(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint64) & np.uint64(0x1249249249249249)
    v = (v ^ (v >> np.uint64(2))) & np.uint64(0x10C30C30C30C30C3)
    v = (v ^ (v >> np.uint64(4))) & np.uint64(0x100F00F00F00F00F)
    v = (v ^ (v >> np.uint64(8))) & np.uint64(0x1F0000FF0000FF)
    v = (v ^ (v >> np.uint64(16))) & np.uint64(0x1F00000000FFFF)
    v = (v ^ (v >> np.uint64(32))) & np.uint64(0x1FFFFF)
    return v


def morton_encode(x, y, z) -> np.ndarray:
    """Interleave x (bit 3k), y (3k+1), z (3k+2); same bit layout as
    Morton_Assist::morton_encode (Morton_Assist.cpp:185-193)."""
    x = np.asarray(x, np.uint64)
    y = np.asarray(y, np.uint64)
    z = np.asarray(z, np.uint64)
    return _dilate3(x) | (_dilate3(y) << np.uint64(1)) | (_dilate3(z) << np.uint64(2))


def morton_decode(k):
    k = np.asarray(k, np.uint64)
    return (_compact3(k).astype(np.int64), _compact3(k >> np.uint64(1)).astype(np.int64),
            _compact3(k >> np.uint64(2)).astype(np.int64))


def cell_key(max_level: int, level: int, x, y, z) -> np.ndarray:
    """Key of the level-`level` cell at integer coordinates (x, y, z) in that
    level's units (the refinement bits below the level are zero)."""
    s = np.uint64(max_level - level)
    return morton_encode(np.asarray(x, np.uint64) << s, np.asarray(y, np.uint64) << s,
                         np.asarray(z, np.uint64) << s)


def cell_coords(max_level: int, level: int, keys):
    x, y, z = morton_decode(keys)
    s = max_level - level
    return x >> s, y >> s, z >> s


def reference_units(nu: float, u_ref: float, max_level: int, c_dx: float = 1.0, u_dt: float = 1.0,
                    collision: str = "LBGK"):
    """Per-level relaxation times and the lattice velocity exactly as
    LBM_Manager::setUnit + checkMach compute them (LBM_Manager.cpp:743-844),
    with the grid spacing dx[l] = c_dx / 2^l set for every level (the
    reference leaves dx[l] = 0 for l < L, Lat_Voxelize.cpp:422; callers here
    always provide it).  Returns (tau[list], CF_U, u_lattice)."""
    max_mach = 0.09
    min_tau = 0.500001
    l_cs = 1.0 / 1.7320508075688772
    l_cssq = 1.0 / 3.0
    lsize = [1.0 / float(1 << l) for l in range(max_level + 1)]
    ltime = [1.0 / float(1 << l) for l in range(max_level + 1)]
    dt0 = u_dt
    if collision == "LBGK":
        for l in range(max_level + 1):
            dx = c_dx * lsize[l]
            dt = dt0 * ltime[l]
            max_dt = dx * max_mach * l_cs / u_ref
            min_dt = dx * dx * (min_tau - 0.5) * l_cssq / nu
            if dt < min_dt or dt > max_dt:
                dt0 = max_dt * 0.99 / ltime[l]
    cf_l = [c_dx * lsize[l] for l in range(max_level + 1)]
    cf_t = [dt0 * ltime[l] for l in range(max_level + 1)]
    cf_u = cf_l[0] / cf_t[0]
    cf_nu = [cf_l[l] * cf_u for l in range(max_level + 1)]
    ma = (u_ref / cf_u) / l_cs
    if ma >= max_mach:
        ref_vel = (u_ref / cf_u) * cf_u
        cf_u = ref_vel / (0.9 * max_mach * l_cs)
        cf_nu = [cf_l[l] * cf_u for l in range(max_level + 1)]
    tau = [nu / cf_nu[l] / l_cssq + 0.5 for l in range(max_level + 1)]
    return tau, cf_u, u_ref / cf_u
