"""Lattice classification on the device (mt_case_generate) against the host
mesher: the same keys, set tags and neighbour tables on every level, and
bit-identical populations and forces after stepping both builds (analytic
spheres, direct-forcing bands and triangulated STL surfaces)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from mortontrie_amr_b200.lbm import Context
    c = Context(0)
    yield c
    c.close()


def _cases():
    from mortontrie_amr_b200.case import (Octree, cavity_case, df_sphere_case, nested_sphere_case, sphere_case,
                                          surface_case, uniform_box_case)
    from mortontrie_amr_b200.stl import box_surface, icosphere
    return {
        "sphere_q19_fh": sphere_case(coarse=(32, 16, 16), refine=[((6, 4, 4), (18, 12, 12))], center=(12, 8, 8),
                                     radius=2.0),
        "sphere_q27_dw": sphere_case(q=27, ib_method="DW", coarse=(30, 18, 18), refine=[((6, 5, 5), (18, 13, 13))],
                                     center=(12, 9, 9), radius=2.0),
        "nested_q27_cumulant_l3": nested_sphere_case(coarse=(64, 32, 32), max_level=3, center=(20, 16, 16),
                                                     radius=2.0, half_widths=(5.0, 3.5, 2.5), re=50.0),
        "cavity_q19_l2": cavity_case(q=19, coarse=(24, 24, 24), max_level=2, re=100.0),
        "cavity_q27_l0": cavity_case(q=27, collision="Cumulant", coarse=(16, 16, 16), max_level=0),
        "df_osc_l2": df_sphere_case(radius=3, max_level=2, re=60.0, oscillating=True, period=100),
        "df_slack_l1": df_sphere_case(radius=4, max_level=1, re=80.0, band_slack=1.0),
        "box_periodic_empty": uniform_box_case(q=19, n=(16, 12, 8), empty_levels=1),
        "surface_icosphere_q19_fh": surface_case(icosphere((12, 8, 8), 2.0, 3), coarse=(32, 16, 16),
                                                 refine=[((6, 4, 4), (18, 12, 12))]),
        "surface_box_q27_dw": surface_case(box_surface((10.3, 6.6, 6.1), (13.7, 9.4, 9.85)), q=27,
                                           collision="Cumulant", ib_method="DW", coarse=(32, 16, 16),
                                           refine=[((6, 4, 4), (18, 12, 12))]),
        "surface_icosphere_l2": surface_case(icosphere((16, 12, 12), 2.0, 3), coarse=(48, 24, 24), max_level=2,
                                             refine=[((8, 6, 6), (26, 18, 18)), ((22, 16, 16), (42, 32, 32))],
                                             re=50.0),
        # refinement made from the body (regions uploaded with mt_case_set_region)
        "octree_sphere_q19_l3": sphere_case(coarse=(48, 24, 24), max_level=3, center=(16, 12, 12), radius=2.5,
                                            octree=Octree()),
        "octree_df_osc_l2": df_sphere_case(radius=3, max_level=2, re=60.0, oscillating=True, period=100,
                                           octree=Octree(band=2.0, margin=4)),
        "octree_surface_q27_l2": surface_case(icosphere((16.3, 12.1, 11.8), 2.5, 3), q=27, collision="Cumulant",
                                              coarse=(48, 24, 24), max_level=2, octree=Octree(band=2.0, margin=5)),
    }


CASES = sorted(_cases())


@pytest.mark.parametrize("name", CASES)
def test_generated_sets_match_host_mesher(ctx, name):
    from mortontrie_amr_b200.lbm import LBM_Manager
    case = _cases()[name]
    a = LBM_Manager(ctx, case, schedule="fused")
    b = LBM_Manager(ctx, case, schedule="fused", generate=True)
    for l in range(case.max_level + 1):
        ka, ta = a.keys(l)
        kb, tb = b.keys(l)
        assert np.array_equal(ka, kb), (name, l, ka.size, kb.size)
        assert np.array_equal(ta, tb), (name, l, int((ta != tb).sum()))
        assert np.array_equal(a.neighbors(l), b.neighbors(l)), (name, l)
    a.fluidSimulate(3)
    b.fluidSimulate(3)
    ctx.synchronize()
    for l in range(case.max_level + 1):
        fa, ca = a.populations(l)
        fb, cb = b.populations(l)
        assert np.array_equal(fa, fb) and np.array_equal(ca, cb), (name, l)
    assert np.array_equal(a.force(), b.force()), name
    a.close()
    b.close()


def test_spec_mesh_case_runs_without_host_sets(ctx):
    """A case made with mesh="device" has no host sets at all and matches
    the host-mesher build step for step."""
    from mortontrie_amr_b200.case import df_sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    from mortontrie_amr_b200.mesh import SpecMesh
    host = df_sphere_case(radius=3, max_level=1, re=50.0, oscillating=True, period=60)
    dev = df_sphere_case(radius=3, max_level=1, re=50.0, oscillating=True, period=60, mesh="device")
    assert isinstance(dev.mesh, SpecMesh)
    a = LBM_Manager(ctx, host, storage="f16", schedule="fused")
    b = LBM_Manager(ctx, dev, storage="f16", schedule="fused")
    a.fluidSimulate(4)
    b.fluidSimulate(4)
    ctx.synchronize()
    for l in range(2):
        assert np.array_equal(a.populations(l)[0], b.populations(l)[0]), l
    assert np.array_equal(a.force(), b.force())
    a.close()
    b.close()


@pytest.mark.parametrize("bad", ["box_touches_bc", "box_near_interface", "solid_near_interface",
                                 "band_near_interface"])
def test_generated_contract_errors_match_host_mesher(ctx, bad):
    """The device raises MT_ERR_MESH where the host mesher raises, with the
    same message."""
    from mortontrie_amr_b200.case import CaseParams, Case
    from mortontrie_amr_b200.lbm import LBM_Manager, MTError
    from mortontrie_amr_b200.mesh import MeshSpec, Sphere, SpecMesh, build_mesh
    sp = {
        "box_touches_bc": MeshSpec(q=19, max_level=1, coarse=(16, 16, 16), refine=[((0, 4, 4), (8, 12, 12))],
                                   boundary=("bc", "bc", "bc")),
        "box_near_interface": MeshSpec(q=19, max_level=2, coarse=(24, 16, 16),
                                       refine=[((4, 4, 4), (16, 12, 12)), ((8, 8, 8), (20, 16, 16))],
                                       boundary=("bc", "periodic", "periodic")),
        "solid_near_interface": MeshSpec(q=19, max_level=1, coarse=(32, 16, 16), refine=[((6, 4, 4), (18, 12, 12))],
                                         boundary=("bc", "periodic", "periodic"), sphere=Sphere((12, 8, 8), 3.6)),
        "band_near_interface": MeshSpec(q=19, max_level=1, coarse=(32, 16, 16), refine=[((6, 4, 4), (18, 12, 12))],
                                        boundary=("bc", "periodic", "periodic"), sphere=Sphere((12, 8, 8), 2.5),
                                        ib="markers"),
    }[bad]
    with pytest.raises(ValueError) as host_err:
        build_mesh(sp)
    ib = "DF" if sp.ib == "markers" else "FH"
    case = Case(SpecMesh(spec=sp), CaseParams(q=19, ib_method=ib, bc_mode="zouhe_outflow"))
    with pytest.raises(MTError) as dev_err:
        LBM_Manager(ctx, case)
    assert "MT_ERR_MESH" in str(dev_err.value)
    host_msg = str(host_err.value).split(": ", 1)[-1]
    assert host_msg in str(dev_err.value), (str(host_err.value), str(dev_err.value))


def test_flow_output_of_a_stepped_case(ctx, tmp_path):
    """write_flow writes the device's velocity of every lat_f and F2C cell
    (tecplot.cpp:16-176 layout) after a few steps."""
    from mortontrie_amr_b200.case import sphere_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    from mortontrie_amr_b200.tecplot import write_flow
    case = sphere_case(coarse=(32, 16, 16), refine=[((6, 4, 4), (18, 12, 12))], center=(12, 8, 8), radius=2.0,
                       mesh="device")
    mgr = LBM_Manager(ctx, case, storage="f32", schedule="fused")
    mgr.fluidSimulate(5)
    ctx.synchronize()
    path = write_flow(mgr, str(tmp_path), 5, u_scale=2.0)
    assert path.endswith("sphereFlow_5.000000.dat")
    lines = open(path).read().splitlines()
    head = dict(kv.split("=") for kv in lines[2].replace("ZONE, ", "").split(", ")[:2])
    n, e = int(head["NODES"]), int(head["ELEMENTS"])
    want = []
    for l in range(mgr.L + 1):
        _, tags = mgr.keys(l)
        _, u = mgr.macros(l)
        sel = np.concatenate([np.flatnonzero(tags & 1), np.flatnonzero(tags & 2)])
        want.append(u[:, sel])
    want = 2.0 * np.concatenate(want, axis=1)
    assert want.shape[1] == e
    got = np.array([float(v) for v in lines[3 + 3 * n:3 + 3 * n + 3 * e]]).reshape(3, e)
    assert np.allclose(got, want, rtol=1e-5, atol=1e-9)
    assert np.abs(want).max() > 1e-3      # the flow has started
    mgr.close()


def test_region_arguments(ctx):
    """mt_case_set_region / mt_case_generate with regions: levels out of
    range, boxes outside the coarser level's extent, regions beside boxes
    and a refined level without its region are refused."""
    import ctypes as C
    from mortontrie_amr_b200.case import Octree, sphere_case
    from mortontrie_amr_b200.lbm import _ptr, lib, make_desc, make_mesh_spec
    case = sphere_case(coarse=(48, 24, 24), max_level=2, center=(16, 12, 12), radius=2.5, octree=Octree(),
                       mesh="device")
    d = make_desc(case, "f64", None)
    cid = C.c_int32()
    assert lib().mt_case_create(ctx.h, C.byref(d), C.byref(cid)) == 0
    lo = np.zeros(3, np.int64)
    shape = np.array([4, 4, 4], np.int64)
    mask = np.ones(64, np.uint8)
    args = lambda l, lo_, sh_: (ctx.h, cid.value, l, _ptr(lo_, C.c_int64), _ptr(sh_, C.c_int64), _ptr(mask, C.c_uint8))
    assert lib().mt_case_set_region(*args(0, lo, shape)) == -1           # level 0 has no region
    assert lib().mt_case_set_region(*args(3, lo, shape)) == -1           # above max_level
    far = np.array([46, 0, 0], np.int64)
    assert lib().mt_case_set_region(*args(1, far, shape)) == -1          # leaves level 0's extent
    assert lib().mt_case_set_region(*args(1, np.array([20, 10, 10], np.int64), shape)) == 0
    ms = make_mesh_spec(case.mesh.spec)
    assert lib().mt_case_generate(ctx.h, cid.value, C.byref(ms)) == -3   # level 2's region missing
    ms.has_refine[1] = 1                                                  # a box beside a region
    assert lib().mt_case_generate(ctx.h, cid.value, C.byref(ms)) == -1
    lib().mt_case_destroy(ctx.h, cid.value)
