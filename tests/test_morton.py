"""Morton neighbour arithmetic against Morton_Assist::find_neighbor known
answers (tests/golden/morton_kat_q27_l2.npz, produced by the reference)."""
import os

import numpy as np
from helpers import GOLDEN_DIR


def test_neighbor_keys_match_reference():
    import oracle as O
    from mortontrie_amr_b200.case import Case, CaseParams
    from mortontrie_amr_b200.mesh import MeshSpec, build_mesh
    z = np.load(os.path.join(GOLDEN_DIR, "morton_kat_q27_l2.npz"))
    # a throw-away case only to carry L = 2, Q = 27 and non-periodic axes
    spec = MeshSpec(q=27, max_level=2, coarse=(4, 4, 4), refine=[None, None], boundary=("bc", "bc", "bc"))
    oc = O.OracleCase(Case(build_mesh(spec), CaseParams(q=27, u_bc=(0.01, 0, 0), u_ref=0.01)))
    for lev in range(3):
        m = z["levels"] == lev
        got = oc.neighbor_keys(lev, z["keys"][m])
        np.testing.assert_array_equal(got, z["neighbors"][m])


def test_encode_decode_roundtrip():
    from mortontrie_amr_b200.lattice import cell_coords, cell_key
    rng = np.random.default_rng(0)
    for L in range(4):
        for l in range(L + 1):
            x, y, z = (rng.integers(0, 1 << (18 - L + l), 500) for _ in range(3))
            k = cell_key(L, l, x, y, z)
            a, b, c = cell_coords(L, l, k)
            assert np.array_equal(a, x) and np.array_equal(b, y) and np.array_equal(c, z)
