"""The CPU oracle against the reference's own multi-dump traces
(tests/golden/*.npz of TRACE_CASES, made by gen_golden.py --trace with the
reference's LBM translation units): bit-exact f on every non-boundary cell,
fcol everywhere, rho and u on lat_f, after the first recorded coarse-step
count of every trace (the later counts, up to cfg1's 1000 coarse steps, are
checked against the GPU path, where they take seconds)."""
import numpy as np
import pytest
from golden_cases import TRACE_CASES
from helpers import init_of, load_trace, oracle_state, rel_err, run_oracle, trace_mismatches


@pytest.mark.parametrize("name", sorted(TRACE_CASES))
def test_oracle_matches_reference_trace(name):
    from gen_golden import set_digest
    spec, case, z, meta = load_trace(name)
    assert set_digest(case) == meta["set_digest"], "mesher output changed; regenerate the goldens"
    n = spec["dumps"][0]
    oc = run_oracle(case, n, init_of(case, spec))
    assert trace_mismatches(case, z, 0, oracle_state(oc)) == []
    force = oc.force()
    ref = z["force"][:n].sum(axis=0)
    assert force[3] == ref[3]
    if np.abs(ref[:3]).max() > 0:
        assert rel_err(force[:3], ref[:3]) < 1e-12


def test_trace_goldens_are_finite():
    """Every recorded state of the reference is finite (a golden of a
    diverged run would pin nothing)."""
    for name, spec in TRACE_CASES.items():
        _, case, z, _ = load_trace(name)
        for d in range(len(spec["dumps"])):
            for l in range(case.max_level + 1):
                assert bool(z[f"finite_{d}_{l}"][0]), (name, d, l)
