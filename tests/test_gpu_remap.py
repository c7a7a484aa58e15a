"""Carrying a state onto another lattice (mt_case_remap): the moving
refinement of a body.  The same lattice gives the same state bit for bit; an
equilibrium stays that equilibrium whichever cells are copied, exploded from
a parent or coalesced from children; a run whose refinement box moves keeps
going from the carried state."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from mortontrie_amr_b200.lbm import Context
    c = Context(0)
    yield c
    c.close()


def _box_case(lo, hi, u=(0.05, 0.0, 0.0)):
    from mortontrie_amr_b200.case import Case, CaseParams
    from mortontrie_amr_b200.mesh import MeshSpec, SpecMesh
    spec = MeshSpec(q=19, max_level=2, coarse=(32, 16, 16),
                    refine=[(lo, hi), tuple(tuple(2 * v + d for v in b) for b, d in zip((lo, hi), (3, -3)))],
                    boundary=("periodic",) * 3)
    return Case(SpecMesh(spec=spec), CaseParams(q=19, nu=0.02, u_bc=u, u_ref=0.05, bc_mode="neq"))


@pytest.mark.parametrize("storage", ["f64", "f16"])
def test_remap_onto_the_same_lattice_is_exact(ctx, storage):
    from mortontrie_amr_b200.case import sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = sphere_case(coarse=(32, 16, 16), refine=[((6, 4, 4), (18, 12, 12))], center=(12, 8, 8), radius=2.0,
                       mesh="device")
    a = LBM_Manager(ctx, case, storage, schedule="fused")
    a.fluidSimulate(5)
    b = a.remeshed(case)
    counts = b.remap_from(a)
    assert counts[:, 1:].sum() == 0 and counts[:, 0].sum() == sum(b.size(l) for l in range(2))
    for l in range(2):
        fa, ca = a.populations(l)
        fb, cb = b.populations(l)
        assert np.array_equal(fa, fb) and np.array_equal(ca, cb), l
    a.fluidSimulate(3)
    b.fluidSimulate(3)
    ctx.synchronize()
    for l in range(2):
        assert np.array_equal(a.populations(l)[0], b.populations(l)[0]), l
    a.close()
    b.close()


def test_equilibrium_survives_a_moved_refinement(ctx):
    """A uniform equilibrium carried onto boxes moved by two coarse cells:
    copied, exploded and coalesced cells all hold the same equilibrium."""
    from mortontrie_amr_b200.case import equilibrium
    from mortontrie_amr_b200.lbm import LBM_Manager
    a = LBM_Manager(ctx, _box_case((8, 4, 4), (20, 12, 12)), "f64")
    b = LBM_Manager(ctx, _box_case((10, 4, 4), (22, 12, 12)), "f64")
    a.initial_equilibrium(1.02, (0.05, 0.01, -0.02))
    counts = b.remap_from(a)
    assert counts[1, 1] > 0 and counts[0, 2] > 0 and counts[1, 2] > 0 and counts[:, 3].sum() == 0
    feq = equilibrium(19, np.array([1.02]), np.array([0.05]), np.array([0.01]), np.array([-0.02]))[:, 0]
    for l in range(3):
        f, fcol = b.populations(l)
        assert np.abs(f - feq[:, None]).max() < 1e-14, l
        assert np.abs(fcol - feq[:, None]).max() < 1e-14, l
    a.close()
    b.close()


@pytest.mark.parametrize("storage", ["f64", "f16"])
def test_run_with_moving_refinement(ctx, storage):
    """A sphere flow whose refinement box follows a shift of the body's
    region: the carried state keeps running and stays close to the run on
    the fixed box away from the interfaces."""
    from mortontrie_amr_b200.case import sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    kw = dict(coarse=(40, 16, 16), center=(14, 8, 8), radius=2.0, re=20.0, mesh="device")
    a = LBM_Manager(ctx, sphere_case(refine=[((6, 4, 4), (20, 12, 12))], **kw), storage, schedule="fused")
    a.fluidSimulate(20)
    b = a.remeshed(sphere_case(refine=[((7, 4, 4), (21, 12, 12))], **kw))
    a.fluidSimulate(10)
    b.fluidSimulate(10)
    ctx.synchronize()
    b.status()
    ka, _ = a.keys(0)
    kb, tb = b.keys(0)
    _, ua = a.macros(0)
    _, ub = b.macros(0)
    common, ia, ib = np.intersect1d(ka, kb, return_indices=True)
    keep = (tb[ib] & 1) != 0
    du = np.linalg.norm(ua[:, ia[keep]] - ub[:, ib[keep]]) / np.linalg.norm(ua[:, ia[keep]])
    assert np.isfinite(du) and du < 0.05, du
    a.close()
    b.close()


def test_moving_refinement_follows_the_sphere(ctx):
    """An oscillating direct-forcing sphere run in windows whose refinement
    and forcing band cover only that window's displacements: the forcing
    steps continue across the re-meshes, the band is smaller than the static
    swept band, and the mean force stays close to the static mesh's."""
    from mortontrie_amr_b200.case import df_sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    from mortontrie_amr_b200.moving import MovingSphere
    kw = dict(radius=3, max_level=2, re=40.0, u=0.1, amplitude=0.5, period=1000)
    static = LBM_Manager(ctx, df_sphere_case(oscillating=True, mesh="device", **kw), "f32", schedule="fused",
                         scaling="standard")
    mv = MovingSphere(ctx, storage="f32", window=4, **kw)
    static.fluidSimulate(24)
    mv.step(24)
    ctx.synchronize()
    fs, fm = static.force(), mv.total_force()
    assert mv.windows == 6
    assert fs[3] == fm[3] == 24 * 4
    assert np.all(np.isfinite(fm))
    band_static = int(np.count_nonzero(static.keys(2)[1] & 256))
    band_moving = int(np.count_nonzero(mv.mgr.keys(2)[1] & 256))
    assert band_moving < band_static
    assert abs(fm[0] - fs[0]) < 0.1 * abs(fs[0]), (fm, fs)
    static.close()
    mv.close()


@pytest.mark.parametrize("scaling", ["reference", "standard"])
def test_remap_matches_cpu_restatement(ctx, scaling):
    """FP64 remap of a perturbed state onto moved boxes equals the CPU
    restatement (oracle.remap_restated) bit for bit, cell kinds included."""
    import oracle as O
    from mortontrie_amr_b200.lbm import LBM_Manager
    a = LBM_Manager(ctx, _box_case((8, 4, 4), (20, 12, 12)), "f64", scaling=scaling)
    b = LBM_Manager(ctx, _box_case((10, 4, 4), (22, 12, 12)), "f64", scaling=scaling)
    rng = np.random.default_rng(11)
    src = []
    for l in range(3):
        f, fcol = a.populations(l)
        f = f * (1.0 + 0.01 * rng.standard_normal(f.shape))
        fcol = fcol * (1.0 + 0.01 * rng.standard_normal(fcol.shape))
        a.set_populations(l, f, fcol)
        keys, tags = a.keys(l)
        src.append((keys, tags, f, fcol))
    counts = b.remap_from(a)
    dst = [b.keys(l) for l in range(3)]
    taus = list(b.case.params.taus(2))
    want = O.remap_restated(19, 2, dst, src, taus, scaling == "standard", b.case.params.rho0, b.case.params.u_bc)
    for l in range(3):
        f, fcol = b.populations(l)
        wf, wc, kind = want[l]
        assert np.array_equal(f, wf), (l, float(np.abs(f - wf).max()))
        assert np.array_equal(fcol, wc), (l, float(np.abs(fcol - wc).max()))
        assert counts[l].tolist() == np.bincount(kind, minlength=4).tolist(), l
    assert counts[:, 1].sum() > 0 and counts[:, 2].sum() > 0
    a.close()
    b.close()
