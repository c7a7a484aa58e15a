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
