"""Morton neighbour arithmetic against Morton_Assist::find_neighbor known
answers (tests/golden/morton_kat_q27_l2.npz, produced by the reference)."""
import os

import numpy as np
import pytest
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


def _blocks(q, L):
    return np.load(os.path.join(GOLDEN_DIR, f"morton_blocks_q{q}_l{L}.npz"))


@pytest.mark.parametrize("q,L", [(19, 1), (19, 3), (27, 3)])
def test_neighbor_keys_match_reference_blocks(q, L):
    """Every cell of two 8^3 blocks per level (the origin and a block
    straddling 32 * 2^l), every direction: the oracle's Morton neighbour
    arithmetic equals Morton_Assist::find_neighbor."""
    import oracle as O
    from mortontrie_amr_b200.case import Case, CaseParams
    from mortontrie_amr_b200.mesh import MeshSpec, build_mesh
    z = _blocks(q, L)
    spec = MeshSpec(q=q, max_level=L, coarse=(4, 4, 4), refine=[None] * L, boundary=("bc", "bc", "bc"))
    oc = O.OracleCase(Case(build_mesh(spec), CaseParams(q=q, u_bc=(0.01, 0, 0), u_ref=0.01)))
    for lev in range(L + 1):
        m = z["levels"] == lev
        np.testing.assert_array_equal(oc.neighbor_keys(lev, z["keys"][m]), z["neighbors"][m])


def blocks_case(q, L):
    """A case whose level-l lat_f set is the KAT blocks' cells of level l and
    every neighbour key the reference gives them (so every link hits)."""
    from mortontrie_amr_b200.case import Case, CaseParams
    from mortontrie_amr_b200.mesh import SET_NAMES, Mesh, MeshSpec
    z = _blocks(q, L)
    levels = []
    for lev in range(L + 1):
        m = z["levels"] == lev
        k = np.unique(np.concatenate([z["keys"][m], z["neighbors"][m].ravel()]))
        sets = {name: np.zeros(0, np.uint64) for name in SET_NAMES}
        sets["lat_f"] = k
        levels.append(sets)
    n0 = 1 << (21 - L)
    spec = MeshSpec(q=q, max_level=L, coarse=(n0, n0, n0), refine=[None] * L, boundary=("bc", "bc", "bc"))
    mesh = Mesh(spec=spec, levels=levels, lat_bc=[np.zeros(0, np.uint64) for _ in range(26)],
                dis_keys=np.zeros(0, np.uint64), dis_rows=np.zeros((0, q - 1)),
                extent=[tuple(n0 << l for _ in range(3)) for l in range(L + 1)])
    return Case(mesh, CaseParams(q=q, u_bc=(0.01, 0, 0), u_ref=0.01)), z
