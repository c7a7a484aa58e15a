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


def _host_info(mgr, prev):
    """infoPrint's quantities from the read-back macros: per level max |u|
    and cells with |u| > 1 over lat_f and F2C, sum |u - prev|^2 and sum |u|^2
    over lat_f (prev: the lat_f velocities of the previous call, or None)."""
    rows, snap = [], []
    for l in range(mgr.L + 1):
        _, u = mgr.macros(l)
        _, tags = mgr.keys(l)
        both = (tags & 3) != 0
        latf = (tags & 1) != 0
        v = np.sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2])
        ul = u[:, latf]
        e2 = 0.0 if prev is None else float(((ul - prev[l]) ** 2).sum())
        rows.append([float(v[both].max()) if both.any() else 0.0, int((v[both] > 1.0).sum()), e2,
                     float((ul * ul).sum())])
        snap.append(ul)
    return np.array(rows), snap


@pytest.mark.parametrize("schedule", ["phases", "fused"])
def test_info_matches_host_diagnostics(ctx, schedule):
    """mt_case_info (the diagnostics LBM_Manager::infoPrint prints) against
    the same quantities from the read-back FP64 macros: the maximum and the
    count exactly, the sums to 1e-12; the velocity change is measured from
    the previous call (zero on the first)."""
    from mortontrie_amr_b200.case import nested_sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = nested_sphere_case(coarse=(48, 24, 24), max_level=2, center=(16, 12, 12), radius=2.0,
                              half_widths=(4.0, 2.5), re=50.0)
    mgr = LBM_Manager(ctx, case, schedule=schedule)
    mgr.fluidSimulate(2)
    d0 = mgr.info()
    h0, snap = _host_info(mgr, None)
    assert np.all(d0[:, 2] == 0)
    mgr.fluidSimulate(1)
    d1 = mgr.info()
    h1, _ = _host_info(mgr, snap)
    for d, h in ((d0, h0), (d1, h1)):
        assert np.array_equal(d[:, 0], h[:, 0]) and np.array_equal(d[:, 1], h[:, 1])
        for c in (2, 3):
            assert np.allclose(d[:, c], h[:, c], rtol=1e-12, atol=0), (c, d[:, c], h[:, c])
    assert d1[:, 2].sum() > 0
    line = mgr.infoPrint(3)
    assert line.startswith("[Iter] 3 Velocity error = ") and "Cd = " in line and " L2=" in line
    mgr.close()
