"""Multi-level FP64 path on the GPU: bit-exact against the reference's golden
vectors and against the CPU oracle, through the C ABI."""
import numpy as np
import pytest
from golden_cases import GOLDEN_CASES
from helpers import TAG_BC, init_of, load_golden, rel_err, run_oracle, sha

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from mortontrie_amr_b200.lbm import Context
    c = Context(0)
    yield c
    c.close()


def _device_case(ctx, case, init, schedule="phases"):
    from mortontrie_amr_b200.lbm import LBM_Manager
    mgr = LBM_Manager(ctx, case, schedule=schedule)
    if init is not None:
        for l, (keys, f) in enumerate(init):
            k, _ = mgr.keys(l)
            assert np.array_equal(k, keys)
            mgr.set_populations(l, f)
    return mgr


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_gpu_matches_reference_goldens(ctx, name):
    spec, case, z, _ = load_golden(name)
    mgr = _device_case(ctx, case, init_of(case, spec))
    mgr.fluidSimulate(spec["steps"])
    ctx.synchronize()
    for l in range(case.max_level + 1):
        keys, tags = mgr.keys(l)
        np.testing.assert_array_equal(keys, z[f"keys{l}"])
        f, fcol = mgr.populations(l)
        keep = (tags & TAG_BC) == 0
        assert np.array_equal(f[:, keep], z[f"f{l}"][:, keep]), (name, l, float(np.abs(f[:, keep] - z[f"f{l}"][:, keep]).max()))
        assert sha(fcol) == bytes(z[f"fcol_sha{l}"]), (name, l)
    force = mgr.force()
    ref = z["force"].sum(axis=0)
    assert force[3] == ref[3]
    if np.abs(ref[:3]).max() > 0:
        assert rel_err(force[:3], ref[:3]) < 1e-12


def test_neighbor_table_matches_oracle(ctx):
    import oracle as O
    from mortontrie_amr_b200.lbm import LBM_Manager
    spec, case, z, _ = load_golden("sphere_q19_dw_l2")
    mgr = LBM_Manager(ctx, case)
    oc = O.OracleCase(case)
    for l in range(case.max_level + 1):
        assert np.array_equal(mgr.neighbors(l), oc.neighbors(l)), l
        keys, _ = mgr.keys(l)
        probe = np.concatenate([keys[::7], keys[::11] + np.uint64(1), np.array([0, 2**63], np.uint64)])
        idx = mgr.find(l, probe)
        want = np.searchsorted(keys, probe)
        want = np.where((want < keys.size) & (keys[np.minimum(want, keys.size - 1)] == probe), want, -1)
        assert np.array_equal(idx, want)


def _cfg1_small(**kw):
    from mortontrie_amr_b200.case import sphere_case
    return sphere_case(coarse=(32, 16, 16), refine=[((6, 4, 4), (18, 12, 12))], center=(12, 8, 8), radius=2.0, **kw)


@pytest.mark.parametrize("steps", [1, 7])
def test_zouhe_outflow_periodic_matches_oracle(ctx, steps):
    """cfg1 boundary set (velocity inlet, outflow, periodic y/z): restated
    boundaries, GPU vs oracle bit-exact."""
    case = _cfg1_small()
    mgr = _device_case(ctx, case, None)
    mgr.fluidSimulate(steps)
    ctx.synchronize()
    oc = run_oracle(case, steps)
    for l in range(2):
        f, fcol = mgr.populations(l)
        g = oc.get(l)
        assert np.array_equal(f, g["f"]) and np.array_equal(fcol, g["fcol"]), l
    assert rel_err(mgr.force()[:3], oc.force()[:3]) < 1e-12


def test_phase_calls_equal_graph_step(ctx):
    """The reference call surface (LBMkernel + calculateMacros issued one by
    one) gives the same state as the graph-replayed coarse step."""
    case = _cfg1_small()
    a = _device_case(ctx, case, None)
    b = _device_case(ctx, case, None)
    a.fluidSimulate(3)
    for _ in range(3):
        b.LBMkernel(0)
        b.calculateMacros()
    ctx.synchronize()
    for l in range(2):
        fa, ca = a.populations(l)
        fb, cb = b.populations(l)
        assert np.array_equal(fa, fb) and np.array_equal(ca, cb)


def test_cfg1_full_size_matches_oracle(ctx):
    """cfg1 at its full size (64x32x32 coarse, 2 levels, sphere R=4) for 10
    coarse steps."""
    from mortontrie_amr_b200.case import sphere_case
    case = sphere_case()
    mgr = _device_case(ctx, case, None)
    mgr.fluidSimulate(10)
    ctx.synchronize()
    oc = run_oracle(case, 10)
    for l in range(2):
        f, fcol = mgr.populations(l)
        g = oc.get(l)
        assert np.array_equal(f, g["f"]), (l, float(np.abs(f - g["f"]).max()))
        assert np.array_equal(fcol, g["fcol"])
    assert rel_err(mgr.force()[:3], oc.force()[:3]) < 1e-12


# relative L2 of the velocity on lat_f cells vs the FP64 path after 30 coarse steps
TOL_AMR = {"f32": 5e-5, "f16": 1e-2, "bf16": 6e-2}


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("which", ["cfg1_q19", "cumulant_q27"])
def test_multilevel_reduced_storage_vs_f64(ctx, storage, which):
    """Multi-level path with FP32 arithmetic on FP32 / FP16 / BF16 stored
    deviations against the FP64 path: velocity field (every level) and drag
    within the stated tolerances."""
    from mortontrie_amr_b200.case import nested_sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    if which == "cfg1_q19":
        case = _cfg1_small()
    else:
        case = nested_sphere_case(coarse=(48, 24, 24), max_level=2, center=(16, 12, 12), radius=2.0,
                                  half_widths=(4.0, 2.5), re=50.0)
    a = LBM_Manager(ctx, case, "f64")
    b = LBM_Manager(ctx, case, storage)
    a.fluidSimulate(30)
    b.fluidSimulate(30)
    ctx.synchronize()
    for l in range(case.max_level + 1):
        _, ua = a.macros(l)
        _, ub = b.macros(l)
        _, tags = a.keys(l)
        fluid = (tags & 1) != 0
        err = np.linalg.norm(ub[:, fluid] - ua[:, fluid]) / np.linalg.norm(ua[:, fluid])
        assert err < TOL_AMR[storage], (which, storage, l, err)
    fa, fb = a.force(), b.force()
    assert fa[3] == fb[3]
    assert abs(fb[0] - fa[0]) / abs(fa[0]) < 10 * TOL_AMR[storage], (fa, fb)


@pytest.mark.parametrize("schedule", ["phases", "fused"])
def test_nonfinite_guard(ctx, schedule):
    """A NaN planted on the host in one population of a lat_f cell (overlap
    cells are rewritten every step) propagates through the steps; the device
    guard reports it as MT_ERR_NONFINITE and the context stays usable."""
    from mortontrie_amr_b200.lbm import MTError
    case = _cfg1_small()
    mgr = _device_case(ctx, case, None, schedule=schedule)
    mgr.fluidSimulate(2)
    assert mgr.status() is None
    f, fcol = mgr.populations(1)
    _, tags = mgr.keys(1)
    fluid = np.flatnonzero((tags & 1) != 0)
    cell = int(fluid[len(fluid) // 3])
    f[3, cell] = np.nan
    mgr.set_populations(1, f, fcol)
    mgr.fluidSimulate(1)
    with pytest.raises(MTError, match="MT_ERR_NONFINITE"):
        mgr.status()
    healthy = _device_case(ctx, case, None)
    healthy.fluidSimulate(1)
    assert healthy.status() is None


def test_missing_child_is_reported(ctx):
    """A contract violation (a coarse F2C cell whose children are not stored)
    returns MT_ERR_MESH instead of faulting, like the reference's .at()
    throwing std::out_of_range."""
    from mortontrie_amr_b200.lbm import LBM_Manager, MTError
    case = _cfg1_small()
    lv1 = case.mesh.levels[1]
    lv1["overlap_C2F"] = lv1["overlap_C2F"][5:]
    with pytest.raises(MTError, match="MT_ERR_MESH"):
        LBM_Manager(ctx, case)


def _nested_small():
    from mortontrie_amr_b200.case import nested_sphere_case
    return nested_sphere_case(coarse=(48, 24, 24), max_level=2, center=(16, 12, 12), radius=2.0,
                              half_widths=(4.0, 2.5), re=50.0)


def _same_state(a, b, L):
    for l in range(L + 1):
        fa, ca = a.populations(l)
        fb, cb = b.populations(l)
        assert np.array_equal(fa, fb), (l, float(np.abs(fa - fb).max()))
        assert np.array_equal(ca, cb), (l, float(np.abs(ca - cb).max()))
        ra, ua = a.macros(l)
        rb, ub = b.macros(l)
        assert np.array_equal(ra, rb) and np.array_equal(ua, ub), l


@pytest.mark.parametrize("schedule", ["fused", "fused_lists"])
@pytest.mark.parametrize("which", ["cfg1_q19", "cumulant_q27", "golden_dw"])
@pytest.mark.parametrize("steps", [1, 2, 5])
def test_fused_schedule_fp64_equals_phases(ctx, which, steps, schedule):
    """The fused schedule (stream of a substep in the same pass as the next
    substep's collision, two post-collision buffers per level) leaves the
    same FP64 state as the reference's phase order after every coarse step:
    populations, macros and the IB force, bit for bit."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    if which == "cfg1_q19":
        case = _cfg1_small()
    elif which == "cumulant_q27":
        case = _nested_small()
    else:
        _, case, _, _ = load_golden("sphere_q19_dw_l2")
    a = LBM_Manager(ctx, case, "f64")
    b = LBM_Manager(ctx, case, "f64", schedule=schedule)
    a.fluidSimulate(steps)
    b.fluidSimulate(steps)
    ctx.synchronize()
    _same_state(a, b, case.max_level)
    fa, fb = a.force(), b.force()
    assert fa[3] == fb[3] and np.array_equal(fa[:3], fb[:3]), (fa, fb)
    # continue from the same state across a level-0 buffer parity change
    a.fluidSimulate(3)
    b.fluidSimulate(3)
    ctx.synchronize()
    _same_state(a, b, case.max_level)


@pytest.mark.parametrize("schedule", ["fused", "fused_lists"])
@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_fused_schedule_matches_goldens(ctx, name, schedule):
    """The reference's golden populations through the fused schedule."""
    spec, case, z, _ = load_golden(name)
    mgr = _device_case(ctx, case, init_of(case, spec), schedule=schedule)
    mgr.fluidSimulate(spec["steps"])
    ctx.synchronize()
    for l in range(case.max_level + 1):
        _, tags = mgr.keys(l)
        f, fcol = mgr.populations(l)
        keep = (tags & TAG_BC) == 0
        assert np.array_equal(f[:, keep], z[f"f{l}"][:, keep]), (name, l)
        assert sha(fcol) == bytes(z[f"fcol_sha{l}"]), (name, l)
    force = mgr.force()
    ref = z["force"].sum(axis=0)
    assert force[3] == ref[3]
    if np.abs(ref[:3]).max() > 0:
        assert rel_err(force[:3], ref[:3]) < 1e-12


def test_fused_schedule_interleaved_with_phase_calls(ctx):
    """Per-phase calls and population writes between fused steps act on the
    current buffers; the next fused step recomputes its lookahead."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = _cfg1_small()
    a = LBM_Manager(ctx, case, "f64")
    b = LBM_Manager(ctx, case, "f64", schedule="fused")
    for m in (a, b):
        m.fluidSimulate(3)
        m.LBMkernel(0)
        m.calculateMacros()
        m.fluidSimulate(2)
    ctx.synchronize()
    _same_state(a, b, case.max_level)
    f, fcol = a.populations(1)
    f = f * (1.0 + 1e-3)
    for m in (a, b):
        m.set_populations(1, f, fcol)
        m.fluidSimulate(2)
    ctx.synchronize()
    _same_state(a, b, case.max_level)
    for sched in ("fused_lists", "phases", "fused"):
        b.set_schedule(sched)
        a.fluidSimulate(2)
        b.fluidSimulate(2)
        ctx.synchronize()
        _same_state(a, b, case.max_level)


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_fused_schedule_reduced_storage_vs_f64(ctx, storage):
    """FP32 arithmetic on stored deviations under the fused schedule, against
    the FP64 phase schedule: same tolerances as the phase schedule."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = _nested_small()
    a = LBM_Manager(ctx, case, "f64")
    b = LBM_Manager(ctx, case, storage, schedule="fused")
    a.fluidSimulate(30)
    b.fluidSimulate(30)
    ctx.synchronize()
    for l in range(case.max_level + 1):
        _, ua = a.macros(l)
        _, ub = b.macros(l)
        _, tags = a.keys(l)
        fluid = (tags & 1) != 0
        err = np.linalg.norm(ub[:, fluid] - ua[:, fluid]) / np.linalg.norm(ua[:, fluid])
        assert err < TOL_AMR[storage], (storage, l, err)
    fa, fb = a.force(), b.force()
    assert fa[3] == fb[3]
    assert abs(fb[0] - fa[0]) / abs(fa[0]) < 10 * TOL_AMR[storage], (fa, fb)


@pytest.mark.parametrize("schedule", ["phases", "fused"])
@pytest.mark.parametrize("q,collision,L", [(19, "LBGK", 1), (27, "Cumulant", 2)])
def test_cavity_matches_oracle(ctx, q, collision, L, schedule):
    """Lid-driven cavity (walls on every face, the Top face strategy moving
    along x, refinement under the lid): GPU FP64 vs the oracle, bit-exact."""
    from mortontrie_amr_b200.case import cavity_case
    case = cavity_case(q=q, collision=collision, coarse=(24, 24, 24), max_level=L, re=100.0)
    mgr = _device_case(ctx, case, None, schedule=schedule)
    mgr.fluidSimulate(6)
    ctx.synchronize()
    oc = run_oracle(case, 6)
    for l in range(L + 1):
        f, fcol = mgr.populations(l)
        _, tags = mgr.keys(l)
        g = oc.get(l)
        # boundary cells' f is only read by their own non-equilibrium sweep,
        # whose in-place order the oracle and the device choose differently
        keep = (tags & TAG_BC) == 0
        assert np.array_equal(f[:, keep], g["f"][:, keep]), (l, float(np.abs(f - g["f"])[:, keep].max()))
        assert np.array_equal(fcol, g["fcol"]), l
    # the lid drives the flow: the cells under it move along +x... or -x
    # under the reference's streaming direction; either way they move
    _, u = mgr.macros(0)
    assert np.abs(u[0]).max() > 1e-3


@pytest.mark.parametrize("schedule", ["phases", "fused", "fused_lists"])
@pytest.mark.parametrize("oscillating", [False, True])
def test_direct_forcing_matches_oracle(ctx, schedule, oscillating):
    """Direct-forcing sphere (Lagrangian markers, 3-point kernel, Guo forcing
    on the band): GPU FP64 vs the oracle, bit-exact populations and macros,
    the same body force up to the order of its FP64 sum."""
    from mortontrie_amr_b200.case import df_sphere_case
    case = df_sphere_case(radius=3, max_level=1, re=50.0, oscillating=oscillating, period=60)
    mgr = _device_case(ctx, case, None, schedule=schedule)
    mgr.fluidSimulate(7)
    ctx.synchronize()
    oc = run_oracle(case, 7)
    for l in range(case.max_level + 1):
        f, fcol = mgr.populations(l)
        _, tags = mgr.keys(l)
        g = oc.get(l)
        keep = (tags & TAG_BC) == 0
        assert np.array_equal(f[:, keep], g["f"][:, keep]), (l, float(np.abs(f - g["f"])[:, keep].max()))
        assert np.array_equal(fcol, g["fcol"]), (l, float(np.abs(fcol - g["fcol"]).max()))
        rho, u = mgr.macros(l)
        assert np.array_equal(rho[keep], g["rho"][keep]), l
    fg, fo = mgr.force(), oc.force()
    assert fg[3] == fo[3] == 14
    assert rel_err(fg[:3], fo[:3]) < 1e-12, (fg, fo)


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_direct_forcing_reduced_storage(ctx, storage):
    from mortontrie_amr_b200.case import df_sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = df_sphere_case(radius=3, max_level=2, re=50.0, oscillating=True, period=200)
    a = LBM_Manager(ctx, case, "f64")
    b = LBM_Manager(ctx, case, storage, schedule="fused")
    a.fluidSimulate(30)
    b.fluidSimulate(30)
    ctx.synchronize()
    L = case.max_level
    _, ua = a.macros(L)
    _, ub = b.macros(L)
    _, tags = a.keys(L)
    fl = (tags & 1) != 0
    err = np.linalg.norm(ub[:, fl] - ua[:, fl]) / np.linalg.norm(ua[:, fl])
    assert err < TOL_AMR[storage], err
    fa, fb = a.force(), b.force()
    assert abs(fb[0] - fa[0]) / abs(fa[0]) < 10 * TOL_AMR[storage], (fa, fb)


@pytest.mark.parametrize("conv", ["reference", "textbook"])
@pytest.mark.parametrize("steps", [1, 7])
def test_zouhe_hh_matches_oracle(ctx, conv, steps):
    """Zou-He / Hecht-Harting inlet and five-population outflow (restated,
    unpinned): GPU vs oracle bit-exact, wall cells included."""
    case = _cfg1_small(bc_mode="zouhe_hh", stream_convention=conv)
    mgr = _device_case(ctx, case, None)
    mgr.fluidSimulate(steps)
    ctx.synchronize()
    oc = run_oracle(case, steps)
    for l in range(2):
        f, fcol = mgr.populations(l)
        g = oc.get(l)
        assert np.array_equal(f, g["f"]) and np.array_equal(fcol, g["fcol"]), (l, float(np.abs(f - g["f"]).max()))
    assert rel_err(mgr.force()[:3], oc.force()[:3]) < 1e-12


def test_zouhe_hh_runs_under_the_phase_schedule_only(ctx):
    from mortontrie_amr_b200.lbm import LBM_Manager, MTError
    mgr = LBM_Manager(ctx, _cfg1_small(bc_mode="zouhe_hh"))
    with pytest.raises(MTError, match="MT_ERR_ARG"):
        mgr.set_schedule("fused")
    mgr.close()


@pytest.mark.parametrize("mode", ["hold", "extrap"])
@pytest.mark.parametrize("schedule", ["phases", "fused"])
def test_interface_hold_matches_oracle(ctx, schedule, mode):
    """Explosion in both substeps (interface_time "hold", or "extrap" from the
    parent state extrapolated to the half step; no reference counterpart):
    GPU FP64 under both schedules vs the oracle, bit-exact."""
    from golden_cases import TRACE_CASES, build_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    import oracle as O
    spec = TRACE_CASES["nested_q19_dw_l3"]
    case = build_case(spec)
    init = init_of(case, spec)
    mgr = LBM_Manager(ctx, case, schedule=schedule, interface_time=mode)
    for l, (_, f) in enumerate(init):
        mgr.set_populations(l, f)
    oc = O.OracleCase(case)
    oc.set_interface_time(mode)
    for l, (_, f) in enumerate(init):
        oc.set_populations(l, f)
    mgr.fluidSimulate(3)
    oc.step(3)
    ctx.synchronize()
    for l in range(case.max_level + 1):
        f, fcol = mgr.populations(l)
        g = oc.get(l)
        keep = (g["tags"] & TAG_BC) == 0
        assert np.array_equal(f[:, keep], g["f"][:, keep]), l
        assert np.array_equal(fcol, g["fcol"]), l
    ref = oc.get(1)["f"]
    oc2 = run_oracle(case, 3, init)
    assert not np.array_equal(oc2.get(1)["f"], ref)   # the option changes the run
    mgr.close()


@pytest.mark.parametrize("storage", ["f16", "f64"])
def test_brick_tuner_keeps_the_trajectory(ctx, storage):
    """mt_case_tune_bricks times the brick pass forms on the case itself and
    leaves the state as it was: a tuned case and an untuned one stay equal
    (FP64 bit for bit; FP16 within the two forms' rounding)."""
    from mortontrie_amr_b200.case import nested_sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = nested_sphere_case(coarse=(48, 24, 24), center=(16, 12, 12), radius=1.5)
    a = LBM_Manager(ctx, case, storage, schedule="fused")
    b = LBM_Manager(ctx, case, storage, schedule="fused")
    a.fluidSimulate(2)
    b.fluidSimulate(2)
    v, ms = a.tune_bricks()
    assert (v >= 0).any() and (ms.max() > 0)
    if storage == "f64":
        assert set(v[v >= 0]) <= {0, 3}  # FP64 has forms 0 and 3 only
        assert (ms[:, [1, 2]] == -1).all()
    a.fluidSimulate(3)
    b.fluidSimulate(3)
    ctx.synchronize()
    for l in range(case.max_level + 1):
        fa, ca = a.populations(l)
        fb, cb = b.populations(l)
        if storage == "f64":
            assert np.array_equal(fa, fb) and np.array_equal(ca, cb), l
        else:
            assert rel_err(ca, cb) < 1e-2, l
    a.close()
    b.close()


def _forms_case(family):
    from mortontrie_amr_b200.case import df_sphere_case, nested_sphere_case, sphere_case
    if family == "cumulant":
        return nested_sphere_case(coarse=(128, 64, 64), max_level=2, center=(40, 32, 32), radius=2.0,
                                  half_widths=(4.0, 2.5), re=50.0)
    if family == "df":
        return df_sphere_case(radius=3, max_level=2, re=50.0, oscillating=True, period=200)
    return sphere_case(coarse=(128, 64, 64), refine=[((36, 24, 24), (60, 40, 40))], center=(48, 32, 32), radius=3.0)


@pytest.mark.parametrize("family,storage", [("cumulant", "f16"), ("cumulant", "f32"), ("cumulant", "bf16"),
                                            ("df", "f16"), ("df", "f32"), ("lbgk", "f16"), ("lbgk", "bf16")])
def test_brick_forms_compute_the_same_values(ctx, family, storage):
    """The one-cell forms of the fused brick pass (0; 2 with more registers;
    3 with the lane's two cells unrolled) share the per-cell arithmetic: a
    case run in each form stays equal to form 0 bit for bit (populations,
    macros, force), boundary cells, partial bricks, the IB level and the
    direct-forcing band included."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = _forms_case(family)
    L = case.max_level
    runs = {}
    for form in (0, 2, 3):
        m = LBM_Manager(ctx, case, storage, schedule="fused")
        m.set_brick_forms([form] * (L + 1))
        m.fluidSimulate(5)
        runs[form] = m
    ctx.synchronize()
    for form in (2, 3):
        _same_state(runs[0], runs[form], L)
        assert np.array_equal(runs[0].force(), runs[form].force()), form
    for m in runs.values():
        m.close()


def test_brick_forms_fp64_and_arguments(ctx):
    """FP64 runs forms 0 and 3 (equal bit for bit); the others, and forms out
    of range, are refused with MT_ERR_ARG."""
    from mortontrie_amr_b200.lbm import LBM_Manager, MTError
    case = _nested_small()
    L = case.max_level
    a = LBM_Manager(ctx, case, "f64", schedule="fused")
    b = LBM_Manager(ctx, case, "f64", schedule="fused")
    b.set_brick_forms([3] * (L + 1))
    for bad in (1, 2, 4):
        with pytest.raises(MTError, match="MT_ERR_ARG"):
            b.set_brick_forms([bad] * (L + 1))
    a.fluidSimulate(3)
    b.fluidSimulate(3)
    ctx.synchronize()
    _same_state(a, b, L)
    c = LBM_Manager(ctx, case, "f16", schedule="fused")
    with pytest.raises(MTError, match="MT_ERR_ARG"):
        c.set_brick_forms([4] * (L + 1))
    c.set_brick_forms([-1] * (L + 1))  # keeps every level's form
    for m in (a, b, c):
        m.close()


@pytest.mark.parametrize("schedule", ["phases", "fused"])
@pytest.mark.parametrize("which", ["sphere_q19_l2", "stl_q27_l2"])
def test_octree_case_matches_oracle(ctx, which, schedule):
    """Refinement made from the body (an octree of 2:1-nested regions around
    an analytic sphere, FH links, or an STL icosphere, D3Q27 cumulant): GPU
    FP64 vs the oracle, bit-exact populations and the drag to 1e-12."""
    from test_octree import _octree_cases
    case = _octree_cases()[which]()
    mgr = _device_case(ctx, case, None, schedule=schedule)
    mgr.fluidSimulate(4)
    ctx.synchronize()
    oc = run_oracle(case, 4)
    for l in range(case.max_level + 1):
        f, fcol = mgr.populations(l)
        _, tags = mgr.keys(l)
        g = oc.get(l)
        keep = (tags & TAG_BC) == 0
        assert np.array_equal(f[:, keep], g["f"][:, keep]), l
        assert np.array_equal(fcol, g["fcol"]), l
    assert rel_err(mgr.force()[:3], oc.force()[:3]) < 1e-12
    mgr.close()


@pytest.mark.parametrize("schedule", ["phases", "fused"])
def test_octree_direct_forcing_matches_oracle(ctx, schedule):
    """A direct-forcing oscillating sphere refined around its forcing band
    (octree, fluid inside on coarser levels): GPU FP64 vs the oracle,
    bit-exact populations and the force to 1e-12."""
    from mortontrie_amr_b200.case import Octree, df_sphere_case
    # period 200 finest steps: the markers move at about 0.2 (a faster path
    # makes this lattice diverge within a few steps)
    case = df_sphere_case(radius=3, max_level=2, re=50.0, oscillating=True, period=200,
                          octree=Octree(band=2.0, margin=4))
    mgr = _device_case(ctx, case, None, schedule=schedule)
    mgr.fluidSimulate(4)
    ctx.synchronize()
    oc = run_oracle(case, 4)
    for l in range(case.max_level + 1):
        f, fcol = mgr.populations(l)
        _, tags = mgr.keys(l)
        g = oc.get(l)
        keep = (tags & TAG_BC) == 0
        assert np.abs(f).max() < 2.0, l  # a physical state
        assert np.array_equal(f[:, keep], g["f"][:, keep]), l
        assert np.array_equal(fcol, g["fcol"]), l
    assert rel_err(mgr.force()[:3], oc.force()[:3]) < 1e-12
    mgr.close()


def test_octree_case_reduced_storage(ctx):
    """The octree sphere in FP16 under the fused schedule against FP64 (1.0e-2
    measured after 20 coarse steps: the octree's interfaces lie within a few
    cells of the body, where the boxes keep them further out)."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    from test_octree import _octree_cases
    case = _octree_cases()["sphere_q19_l2"]()
    a = LBM_Manager(ctx, case, "f64")
    b = LBM_Manager(ctx, case, "f16", schedule="fused")
    a.fluidSimulate(20)
    b.fluidSimulate(20)
    ctx.synchronize()
    L = case.max_level
    _, ua = a.macros(L)
    _, ub = b.macros(L)
    _, tags = a.keys(L)
    fl = (tags & 1) != 0
    assert np.linalg.norm(ub[:, fl] - ua[:, fl]) / np.linalg.norm(ua[:, fl]) < 2 * TOL_AMR["f16"]
    a.close()
    b.close()


@pytest.mark.parametrize("q,L", [(19, 1), (19, 3), (27, 3)])
def test_device_neighbor_table_matches_reference_blocks(ctx, q, L):
    """The device-built neighbour table of the KAT blocks (every cell of two
    8^3 blocks per level, with every neighbour the reference gives them
    stored): each link is the index of the key Morton_Assist::find_neighbor
    returns (the reference's pull direction, +e_q)."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    from test_morton import blocks_case
    case, z = blocks_case(q, L)
    mgr = LBM_Manager(ctx, case)
    for lev in range(L + 1):
        keys, _ = mgr.keys(lev)
        nb = mgr.neighbors(lev)
        m = z["levels"] == lev
        idx = np.searchsorted(keys, z["keys"][m])
        assert np.array_equal(keys[idx], z["keys"][m])
        want = np.searchsorted(keys, z["neighbors"][m][:, 1:])          # (cells, Q-1)
        assert np.array_equal(nb[:, idx].T, want), lev
    mgr.close()


@pytest.mark.parametrize("schedule", ["phases", "fused"])
@pytest.mark.parametrize("name", ["collide_q19_lbgk", "collide_q27_cumulant", "collide_q27_lbgk"])
def test_single_cell_collision_matches_reference(ctx, name, schedule):
    """Single-cell collision known answers from the reference's own
    Collision_LBGK / Collision_Cumulant (seeded cell states, one coarse
    step): the GPU's FP64 post-collision populations of the 64 sampled
    cells, bit for bit."""
    from test_oracle_golden import _collide_kat
    from mortontrie_amr_b200.lbm import LBM_Manager
    z, case, init, idx = _collide_kat(name)
    mgr = LBM_Manager(ctx, case, schedule=schedule)
    keys, _ = mgr.keys(0)
    assert np.array_equal(keys, init[0][0])
    mgr.set_populations(0, init[0][1])
    mgr.fluidSimulate(1)
    ctx.synchronize()
    _, fcol = mgr.populations(0)
    assert np.array_equal(fcol[:, idx], z["fcol"])
    mgr.close()


@pytest.mark.parametrize("which,storage", [("cumulant", "f64"), ("df", "f64"), ("cumulant", "f16")])
def test_checkpoint_resume_equals_continuous(ctx, tmp_path, which, storage):
    """save_checkpoint after 3 coarse steps, load into a fresh case of the
    same lattice, 3 more steps: the same populations and force as 6 steps
    without a break (bit for bit, the direct-forcing markers' path phase
    included); a checkpoint of another lattice is refused."""
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = _forms_case(which) if which == "df" else _nested_small()
    a = LBM_Manager(ctx, case, storage, schedule="fused")
    a.fluidSimulate(3)
    path = str(tmp_path / "state.npz")
    a.save_checkpoint(path)
    assert a.steps() == 3
    a.reset_force()
    a.fluidSimulate(3)
    b = LBM_Manager(ctx, case, storage, schedule="fused")
    b.load_checkpoint(path)
    assert b.steps() == 3
    b.fluidSimulate(3)
    ctx.synchronize()
    _same_state(a, b, case.max_level)
    assert np.array_equal(a.force(), b.force())
    from mortontrie_amr_b200.case import cavity_case
    other = LBM_Manager(ctx, cavity_case(coarse=(16, 16, 16), max_level=1), storage, schedule="fused")
    with pytest.raises(ValueError):
        other.load_checkpoint(path)
    for m in (a, b, other):
        m.close()
