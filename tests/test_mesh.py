"""Invariants of the index-set contract the mesher emits
(Lat_Manager.hpp:245-316 semantics)."""
import numpy as np

from mortontrie_amr_b200.case import sphere_case
from mortontrie_amr_b200.lattice import cell_coords, cell_key


def _cfg1():
    return sphere_case()  # 64x32x32, L=1, sphere R=4 at (16,16,16)


def test_sets_disjoint_and_children_present():
    c = _cfg1()
    m = c.mesh
    L = m.spec.max_level
    for l in range(L + 1):
        s = m.levels[l]
        names = ["lat_f", "overlap_F2C", "overlap_C2F", "ghost_overlap_C2F", "lat_sf"]
        for i, a in enumerate(names):
            for b in names[i + 1:]:
                assert not np.intersect1d(s[a], s[b]).size, (l, a, b)
        assert np.all(np.isin(s["ghost_overlap_F2C"], s["lat_f"]))
    # every child of a coarse F2C cell is a fine C2F cell
    f2c = m.levels[0]["overlap_F2C"]
    x, y, z = cell_coords(L, 0, f2c)
    kids = np.concatenate([cell_key(L, 1, 2 * x + dx, 2 * y + dy, 2 * z + dz)
                           for dx in (0, 1) for dy in (0, 1) for dz in (0, 1)])
    assert np.array_equal(np.unique(kids), m.levels[1]["overlap_C2F"])


def test_sphere_links_and_counts():
    c = _cfg1()
    m = c.mesh
    assert np.all(np.isin(m.dis_keys, m.levels[1]["lat_f"]))
    assert np.all((m.dis_rows == -1.0) | ((m.dis_rows >= 0.0) & (m.dis_rows <= 1.0)))
    assert m.dis_keys.size > 0 and m.levels[1]["lat_sf"].size > 0
    # West/East faces only (y and z periodic)
    assert m.lat_bc[0].size == 32 * 32 and m.lat_bc[1].size == 32 * 32
    assert sum(b.size for b in m.lat_bc[2:]) == 0


def test_window_case_covers_its_displacements():
    """A moving-refinement window: its band covers every marker stencil of
    the window's path positions, it is smaller than the static swept band,
    and its markers follow the whole path like the static case's."""
    from mortontrie_amr_b200.case import df_sphere_case
    from mortontrie_amr_b200.lattice import cell_coords
    from mortontrie_amr_b200.moving import path_window
    L, period = 2, 400
    static = df_sphere_case(radius=3, max_level=L, oscillating=True, period=period)
    t0, t1 = 40, 72
    lo, hi = path_window(t0, t1, 1.5, period)
    assert lo < hi and hi <= 1.5
    win = df_sphere_case(radius=3, max_level=L, oscillating=True, period=period, window=(lo, hi))
    assert win.mesh.levels[L]["ib_band"].size < static.mesh.levels[L]["ib_band"].size
    assert np.array_equal(win.mesh.markers.path, static.mesh.markers.path)
    assert np.array_equal(win.mesh.markers.ref, static.mesh.markers.ref)
    bx, by, bz = cell_coords(L, L, win.mesh.levels[L]["ib_band"])
    band = set(zip(bx.tolist(), by.tolist(), bz.tolist()))
    mk = win.mesh.markers
    c = np.array(mk.center)
    for t in (t0, (t0 + t1) // 2, t1):
        pos = c[:, None] + mk.path[t % period, :3, None] + mk.ref
        base = np.floor(pos).astype(int)
        for d in np.ndindex(3, 3, 3):
            cells = base + (np.array(d) - 1)[:, None]
            assert all(tuple(x) in band for x in cells.T[::53])
