"""Storage shift of the reduced storages (mt_case_desc.u_shift, per level):
FP32 / FP16 / BF16 keep f_k - feq_k(1, u_s).  The default (u_s = 0) is the
f - w_q form; a shift at the inlet velocity keeps the stored deviations small
in a channel flow, on every level or on the levels below the finest (whose
wall populations stay near w).  Full populations read back, the interface
transfers between levels of different shifts, remaps between shifts,
batches of cases with different shifts and the argument checks."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from mortontrie_amr_b200.lbm import Context
    c = Context(0)
    yield c
    c.close()


def _nested():
    from mortontrie_amr_b200.case import nested_sphere_case
    return nested_sphere_case(coarse=(48, 24, 24), max_level=2, center=(16, 12, 12), radius=2.0,
                              half_widths=(4.0, 2.5), re=50.0)


def _df():
    from mortontrie_amr_b200.case import df_sphere_case
    return df_sphere_case(radius=3, max_level=2, re=50.0, oscillating=True, period=200)


def _u_err(a, b, levels):
    out = []
    for l in levels:
        _, ua = a.macros(l)
        _, ub = b.macros(l)
        _, tags = a.keys(l)
        fl = (tags & 1) != 0
        out.append(float(np.linalg.norm(ub[:, fl] - ua[:, fl]) / np.linalg.norm(ua[:, fl])))
    return out


@pytest.mark.parametrize("shift", ["inlet", "far_field"])
@pytest.mark.parametrize("which,schedule", [("cumulant_q27", "phases"), ("cumulant_q27", "fused"),
                                            ("df_q19", "fused")])
def test_inlet_shift_fp16_vs_f64(ctx, which, schedule, shift):
    """FP16 storage shifted at the inlet velocity (every level, or below the
    finest) against the FP64 path after 30 coarse steps: velocity (relative
    L2) within 1e-2 like the unshifted form; with the shift on every level no
    worse than it (the flow is near u_bc almost everywhere, so the stored
    deviations shrink)."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = _nested() if which == "cumulant_q27" else _df()
    L = case.max_level
    levels = range(L + 1) if which == "cumulant_q27" else [L]
    a = LBM_Manager(ctx, case, "f64")
    b = LBM_Manager(ctx, case, "f16", schedule=schedule)
    c = LBM_Manager(ctx, case, "f16", schedule=schedule, storage_shift=shift)
    for m in (a, b, c):
        m.fluidSimulate(30)
    ctx.synchronize()
    eb = _u_err(a, b, levels)
    assert np.all(np.isfinite(eb)), eb
    ec = _u_err(a, c, levels)
    assert max(ec) < 1e-2, (eb, ec)
    if shift == "inlet":
        assert max(ec) <= max(eb), (eb, ec)
    # far_field: which levels gain depends on how far the intermediate levels
    # reach from the body (here level 1 lies close around it and loses)
    fa, fc = a.force(), c.force()
    assert fa[3] == fc[3]
    assert abs(fc[0] - fa[0]) / abs(fa[0]) < 0.1, (fa, fc)
    for m in (a, b, c):
        m.close()


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_full_populations_read_back(ctx, storage):
    """populations() returns full values whatever the shift: after the
    initial equilibrium both shifts agree with FP64 to the storage's rounding
    (half a unit in the last place at 1/3, the largest stored magnitude: the
    solid cells hold -s_k)."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = _nested()
    a = LBM_Manager(ctx, case, "f64")
    b = LBM_Manager(ctx, case, storage)
    c = LBM_Manager(ctx, case, storage, storage_shift=[(0.05, 0.0, 0.0), (0.0, 0.0, 0.0), (0.02, 0.01, 0.0)])
    ctx.synchronize()
    tol = {"f32": 1e-7, "f16": 1.3e-4, "bf16": 1.1e-3}[storage]
    for l in range(case.max_level + 1):
        fa, _ = a.populations(l)
        fb, _ = b.populations(l)
        fc, _ = c.populations(l)
        assert np.max(np.abs(fb - fa)) < tol
        assert np.max(np.abs(fc - fa)) < tol
    for m in (a, b, c):
        m.close()


def test_remap_between_shifts(ctx):
    """A remap onto the same lattice with other shifts converts the stored
    values level by level: the full populations agree to FP16 roundings, and
    the same shift copies the stored values exactly."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = _nested()
    src = LBM_Manager(ctx, case, "f16", schedule="fused", storage_shift="far_field")
    src.fluidSimulate(10)
    same = LBM_Manager(ctx, case, "f16", schedule="fused", storage_shift="far_field")
    other = LBM_Manager(ctx, case, "f16", schedule="fused", storage_shift=[(0, 0, 0), (0.04, 0, 0), (0.04, 0, 0)])
    same.remap_from(src, counts=False)
    other.remap_from(src, counts=False)
    ctx.synchronize()
    for l in range(case.max_level + 1):
        fs, cs = src.populations(l)
        f1, c1 = same.populations(l)
        f2, c2 = other.populations(l)
        assert np.array_equal(fs, f1) and np.array_equal(cs, c1)
        # two FP16 roundings apart at most (solid cells: -s_0 and -w_0, near 1/3)
        assert np.max(np.abs(f2 - fs)) < 2.5e-4 and np.max(np.abs(c2 - cs)) < 2.5e-4
    for m in (src, same, other):
        m.close()


def test_batch_groups_by_shift(ctx):
    """Members with different shifts run in separate batched passes; each
    ends where it ends stepped alone."""
    from mortontrie_amr_b200.lbm import Batch, LBM_Manager
    cases = [_df(), _df(), _nested()]
    shifts = [None, "inlet", "far_field"]
    alone = [LBM_Manager(ctx, c, "f16", schedule="fused", storage_shift=s) for c, s in zip(cases, shifts)]
    members = [LBM_Manager(ctx, c, "f16", storage_shift=s) for c, s in zip(cases, shifts)]
    batch = Batch(ctx, members)
    for m in alone:
        m.fluidSimulate(4)
    batch.step(4)
    ctx.synchronize()
    for a, m in zip(alone, members):
        for l in range(a.L + 1):
            for x, y in zip(a.populations(l), m.populations(l)):
                np.testing.assert_allclose(x, y, rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(a.force(), m.force(), rtol=1e-6, atol=1e-9)
    # the two direct-forcing members differ only in their shift
    d = np.max(np.abs(members[0].populations(2)[0] - members[1].populations(2)[0]))
    assert 0.0 < d < 1e-3
    batch.close()
    for m in alone:
        m.close()


def test_shift_arguments(ctx):
    from mortontrie_amr_b200.lbm import LBM_Manager, MTError
    with pytest.raises(MTError, match="MT_ERR_ARG"):
        LBM_Manager(ctx, _nested(), "f16", storage_shift=(0.6, 0.0, 0.0))
    with pytest.raises(MTError, match="MT_ERR_ARG"):
        LBM_Manager(ctx, _nested(), "f16", storage_shift=[(0.0, 0.0, 0.0), (0.0, float("nan"), 0.0), (0, 0, 0)])
    with pytest.raises(ValueError):
        LBM_Manager(ctx, _nested(), "f16", storage_shift="outlet")
    with pytest.raises(ValueError):
        LBM_Manager(ctx, _nested(), "f16", storage_shift=[(0.0, 0.0, 0.0)] * 2)
    # FP64 stores full populations: the shift changes nothing
    a = LBM_Manager(ctx, _nested(), "f64")
    b = LBM_Manager(ctx, _nested(), "f64", storage_shift="inlet")
    a.fluidSimulate(3)
    b.fluidSimulate(3)
    ctx.synchronize()
    for l in range(a.L + 1):
        assert np.array_equal(a.populations(l)[0], b.populations(l)[0])
    a.close()
    b.close()


@pytest.mark.parametrize("schedule", ["phases", "fused"])
def test_level_shifts_across_interfaces(ctx, schedule):
    """Explosion, coalescence and the fused coalescence + collision read one
    level under its shift and write the other under its own: FP32 storage
    with three different level shifts stays within FP32 rounding of the
    unshifted FP32 run (both against FP64)."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = _nested()
    a = LBM_Manager(ctx, case, "f64")
    b = LBM_Manager(ctx, case, "f32", schedule=schedule)
    c = LBM_Manager(ctx, case, "f32", schedule=schedule,
                    storage_shift=[(0.04, 0.0, 0.0), (0.0, 0.02, 0.0), (0.01, 0.0, -0.01)])
    for m in (a, b, c):
        m.fluidSimulate(10)
    ctx.synchronize()
    eb = _u_err(a, b, range(case.max_level + 1))
    ec = _u_err(a, c, range(case.max_level + 1))
    assert max(eb) < 5e-5 and max(ec) < 5e-5, (eb, ec)
    fa, fc = a.force(), c.force()
    assert abs(fc[0] - fa[0]) / abs(fa[0]) < 5e-4, (fa, fc)
    for m in (a, b, c):
        m.close()


def test_moving_refinement_with_level_shifts(ctx):
    """Re-meshing windows of an oscillating direct-forcing sphere with a
    far-field shift (remaps between lattices whose levels carry different
    shifts from the cells they read): the force follows the unshifted FP32
    run to FP32 rounding."""
    from mortontrie_amr_b200.moving import MovingSphere
    kw = dict(radius=3, max_level=2, re=40.0, u=0.1, amplitude=0.5, period=1000)
    a = MovingSphere(ctx, storage="f32", window=4, **kw)
    b = MovingSphere(ctx, storage="f32", window=4, storage_shift="far_field", **kw)
    a.step(12)
    b.step(12)
    ctx.synchronize()
    fa, fb = a.total_force(), b.total_force()
    assert b.windows == 3 and fa[3] == fb[3]
    assert np.all(np.isfinite(fb))
    assert abs(fb[0] - fa[0]) < 1e-4 * abs(fa[0]), (fa, fb)
    a.close()
    b.close()
