"""The CPU oracle against the reference's own outputs (golden vectors made by
tests/golden/gen_golden.py with the reference harness): bit-exact
populations on every stored non-boundary cell, bit-exact post-collision
populations everywhere, drag within 1e-12 (summation order differs)."""
import numpy as np
import pytest
from golden_cases import GOLDEN_CASES
from helpers import TAG_BC, init_of, load_golden, rel_err, run_oracle, sha


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_oracle_matches_reference(name):
    from gen_golden import set_digest
    spec, case, z, meta = load_golden(name)
    assert set_digest(case) == meta["set_digest"], "mesher output changed; regenerate the goldens"
    oc = run_oracle(case, spec["steps"], init_of(case, spec))
    for l in range(case.max_level + 1):
        g = oc.get(l)
        np.testing.assert_array_equal(g["keys"], z[f"keys{l}"])
        keep = (g["tags"] & TAG_BC) == 0
        assert np.array_equal(g["f"][:, keep], z[f"f{l}"][:, keep]), f"level {l} f differs"
        assert sha(g["fcol"]) == bytes(z[f"fcol_sha{l}"]), f"level {l} fcol differs"
    force = oc.force()
    ref = z["force"].sum(axis=0)
    assert force[3] == ref[3]
    if np.abs(ref[:3]).max() > 0:
        assert rel_err(force[:3], ref[:3]) < 1e-12


def test_taus_match_reference_unit_conversion():
    for name in GOLDEN_CASES:
        spec, case, z, _ = load_golden(name)
        assert np.array_equal(np.array(case.params.taus(case.max_level)), z["tau"]), name


def _collide_kat(name):
    import json
    import os
    from golden_cases import COLLIDE_CASES, collide_case, collide_sample, collide_state
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    case = collide_case(COLLIDE_CASES[name])
    init = collide_state(case, meta["seed"])
    idx = collide_sample(case, meta["seed"])
    assert np.array_equal(case.mesh.all_keys(0)[idx], z["keys"])
    assert np.array_equal(init[0][1][:, idx], z["f_in"])  # the same seeded inputs
    return z, case, init, idx


@pytest.mark.parametrize("name", ["collide_q19_lbgk", "collide_q27_cumulant", "collide_q27_lbgk"])
def test_oracle_single_cell_collision(name):
    """Single-cell collision known answers (seeded cell states, rho in
    [0.9, 1.1), |u| < 0.1, a non-equilibrium part; the reference's own
    Collision_LBGK / Collision_Cumulant, Collision_Manager.cpp:13-53 and
    Collision_Cumulant.cpp:22-652): the oracle's post-collision populations
    of the 64 sampled cells, bit for bit."""
    z, case, init, idx = _collide_kat(name)
    oc = run_oracle(case, 1, init[:1] + [init[1]])
    assert np.array_equal(oc.get(0)["fcol"][:, idx], z["fcol"])


@pytest.mark.parametrize("name", ["tgv_q19_32_periodic", "tgv_q27_cumulant_16_periodic", "tgv_q27_lbgk_16_periodic"])
def test_oracle_matches_reference_periodic_tgv(name):
    """The uniform periodic Taylor-Green box (the dense path's workload)
    after 10 steps of the reference's own code (the periodic harness): the
    oracle's f and fcol over every cell, bit for bit."""
    import os
    from golden_cases import TGV_CASES, tgv_reference_case
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    spec = TGV_CASES[name]
    case, init = tgv_reference_case(spec)
    oc = run_oracle(case, spec["steps"], init)
    g = oc.get(0)
    assert sha(g["f"]) == bytes(z["fsha"]) and sha(g["fcol"]) == bytes(z["fcolsha"])
