"""Batches of independent multi-level cases (mt_batch_*): every member of a
batch ends each coarse step in the state it reaches stepped alone, whatever
the mix (models, levels, boundaries, brick or list levels), membership
changes and buffer parities."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from mortontrie_amr_b200.lbm import Context
    c = Context(0)
    yield c
    c.close()


def _mix():
    from mortontrie_amr_b200.case import cavity_case, df_sphere_case, nested_sphere_case, sphere_case
    return [
        sphere_case(coarse=(32, 16, 16), refine=[((6, 4, 4), (18, 12, 12))], center=(12, 8, 8), radius=2.0),
        nested_sphere_case(coarse=(48, 24, 24), max_level=2, center=(16, 12, 12), radius=2.0, half_widths=(4.0, 2.5),
                           re=50.0),
        cavity_case(q=19, coarse=(24, 24, 24), max_level=1, re=100.0),
        cavity_case(q=27, collision="Cumulant", coarse=(24, 24, 24), max_level=2, re=60.0),
        # periodic extent 18 is not a multiple of 4: level 0 runs from cell lists
        sphere_case(coarse=(30, 18, 18), refine=[((6, 5, 5), (18, 13, 13))], center=(12, 9, 9), radius=2.0),
        # direct-forcing oscillating sphere (Lagrangian markers)
        df_sphere_case(radius=3, max_level=2, re=60.0, oscillating=True, period=100),
    ]


def _state(mgr):
    out = []
    for l in range(mgr.L + 1):
        f, fcol = mgr.populations(l)
        rho, u = mgr.macros(l)
        out.append((f, fcol, rho, u))
    return out, mgr.force()


def _assert_same(a, b, exact=True):
    (sa, fa), (sb, fb) = a, b
    for la, lb in zip(sa, sb):
        for x, y in zip(la, lb):
            if exact:
                assert np.array_equal(x, y), float(np.nanmax(np.abs(x - y)))
            else:
                np.testing.assert_allclose(x, y, rtol=1e-6, atol=1e-7)
    if exact:
        assert np.array_equal(fa, fb)
    else:
        np.testing.assert_allclose(fa, fb, rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("storage", ["f64", "f16"])
def test_batch_members_equal_alone(ctx, storage):
    from mortontrie_amr_b200.lbm import Batch, LBM_Manager
    cases = _mix()
    alone = [LBM_Manager(ctx, c, storage, schedule="fused") for c in cases]
    members = [LBM_Manager(ctx, c, storage) for c in cases]
    batch = Batch(ctx, members)
    assert len(batch) == len(cases)
    for m in alone:
        m.fluidSimulate(5)
    batch.step(2)
    batch.step(3)
    ctx.synchronize()
    for a, m in zip(alone, members):
        _assert_same(_state(a), _state(m), exact=(storage == "f64"))
    batch.close()


def test_batch_matches_phase_schedule_fp64(ctx):
    """FP64 members equal the reference's phase order stepped alone."""
    from mortontrie_amr_b200.lbm import Batch, LBM_Manager
    cases = _mix()[:4]
    ref = [LBM_Manager(ctx, c, "f64") for c in cases]
    members = [LBM_Manager(ctx, c, "f64") for c in cases]
    batch = Batch(ctx, members)
    for m in ref:
        m.fluidSimulate(4)
    batch.step(4)
    ctx.synchronize()
    for a, m in zip(ref, members):
        _assert_same(_state(a), _state(m))
    batch.close()


def test_batch_membership_and_parity(ctx):
    """Members join at different coarse-step parities and leave mid-run; the
    others carry on unaffected; a member cannot be stepped on its own."""
    from mortontrie_amr_b200.lbm import Batch, LBM_Manager, MTError
    cases = _mix()
    alone = [LBM_Manager(ctx, c, "f64", schedule="fused") for c in cases[:3]]
    m = [LBM_Manager(ctx, c, "f64", schedule="fused") for c in cases[:3]]
    m[1].fluidSimulate(1)           # odd parity before joining
    alone[1].fluidSimulate(1)
    batch = Batch(ctx, [m[0], m[1]])
    batch.step(3)
    for a in alone[:2]:
        a.fluidSimulate(3)
    with pytest.raises(MTError, match="MT_ERR_STATE"):
        m[0].fluidSimulate(1)
    batch.add(m[2])
    batch.step(2)
    for a in alone:
        a.fluidSimulate(2)
    batch.remove(m[0])
    batch.step(1)
    for a in alone[1:]:
        a.fluidSimulate(1)
    m[0].fluidSimulate(1)           # alone again
    alone[0].fluidSimulate(1)
    ctx.synchronize()
    for a, x in zip(alone, m):
        _assert_same(_state(a), _state(x))
    batch.close()


@pytest.mark.parametrize("storage", ["f64", "f16"])
def test_large_member_runs_its_own_pass(ctx, storage):
    """A member whose level holds 8192 bricks or more (here both levels of a
    96^3 cavity: 706,536 and 1,729,792 cells) runs its own brick pass beside
    the batched pass of the small members; every member still equals itself
    stepped alone."""
    from mortontrie_amr_b200.case import cavity_case
    from mortontrie_amr_b200.lbm import Batch, LBM_Manager
    cases = [cavity_case(q=19, coarse=(96, 96, 96), max_level=1, re=100.0, mesh="device")] + _mix()[:2]
    alone = [LBM_Manager(ctx, c, storage, schedule="fused") for c in cases]
    members = [LBM_Manager(ctx, c, storage) for c in cases]
    assert members[0].size(0) >= 8192 * 64
    batch = Batch(ctx, members)
    for m in alone:
        m.fluidSimulate(3)
    batch.step(3)
    ctx.synchronize()
    for a, m in zip(alone, members):
        _assert_same(_state(a), _state(m), exact=(storage == "f64"))
    batch.close()
    for m in alone + members:
        m.close()
