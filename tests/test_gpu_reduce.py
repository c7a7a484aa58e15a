"""FP64 device reductions of multi-level cases (mt_case_reduce_levels,
mt_case_reduce) against sums of the CPU oracle's populations: per level
over lat_f and overlap_F2C, and the volume-weighted total, within 1e-12
(the summation order differs)."""
import numpy as np
import pytest
from helpers import init_of, load_trace, run_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from mortontrie_amr_b200.lbm import Context
    c = Context(0)
    yield c
    c.close()


def host_rows(case, level_f):
    """rows (L+2, 5) from per-level FP64 populations f (Q, n) in key order"""
    from mortontrie_amr_b200.lattice import directions
    ex, ey, ez, _ = directions(case.q)
    L = case.max_level
    rows = np.zeros((L + 2, 5))
    for l in range(L + 1):
        keys = case.mesh.all_keys(l)
        sel = np.isin(keys, case.mesh.levels[l]["lat_f"]) | np.isin(keys, case.mesh.levels[l]["overlap_F2C"])
        f = level_f(l)[:, sel]
        r = f.sum(axis=0)
        j = np.stack([(f * e[:, None]).sum(axis=0) for e in (ex, ey, ez)])
        rows[l, 0] = r.sum()
        rows[l, 1:4] = j.sum(axis=1)
        rows[l, 4] = (0.5 * (j * j).sum(axis=0) / r).sum()
        rows[L + 1] += rows[l] * 0.125 ** l
    return rows


def _close(got, want, tol):
    scale = np.maximum(np.abs(want[:, :1]), 1.0)  # momentum sums are judged against the mass
    assert np.all(np.abs(got - want) <= tol * np.maximum(np.abs(want), scale)), (got, want)


@pytest.mark.parametrize("schedule", ["phases", "fused"])
def test_reduce_levels_matches_oracle_fp64(ctx, schedule):
    from mortontrie_amr_b200.lbm import LBM_Manager
    spec, case, z, _ = load_trace("nested_q19_dw_l3")
    mgr = LBM_Manager(ctx, case, schedule=schedule)
    init = init_of(case, spec)
    for l, (_, f) in enumerate(init):
        mgr.set_populations(l, f)
    oc = run_oracle(case, 0, init)
    for steps in (1, 3):
        mgr.fluidSimulate(steps)
        oc.step(steps)
        got = mgr.reduce_levels()
        want = host_rows(case, lambda l: oc.get(l)["f"])
        _close(got, want, 1e-12)
        total = np.zeros(5)
        from mortontrie_amr_b200.lbm import lib, _ptr
        import ctypes as C
        ctx.check(lib().mt_case_reduce(ctx.h, mgr.id, _ptr(total, C.c_double)), "reduce")
        np.testing.assert_array_equal(total, got[-1])
    # the same call twice gives the same bits (fixed summation order)
    np.testing.assert_array_equal(mgr.reduce_levels(), mgr.reduce_levels())
    mgr.close()


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_reduce_levels_reduced_storage(ctx, storage):
    """Reduced storages: the FP64 sums of the stored deviations plus the
    shift equal the sums of the populations read back (which add the shift
    in FP32), to the read-back's rounding."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    spec, case, z, _ = load_trace("nested_q19_dw_l3")
    mgr = LBM_Manager(ctx, case, storage=storage, schedule="fused")
    mgr.fluidSimulate(4)
    got = mgr.reduce_levels()
    want = host_rows(case, lambda l: mgr.populations(l)[0])
    _close(got, want, 1e-6)
    mgr.close()
