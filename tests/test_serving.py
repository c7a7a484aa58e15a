"""Host side of the request loop: the seeded Poisson stream, template keys,
per-request cases on shared template meshes and their memory footprint."""
import numpy as np


def test_poisson_stream_is_seeded_and_in_range():
    from mortontrie_amr_b200.serving import poisson_requests
    a = poisson_requests(seed=5, rate=20.0, duration=30.0)
    b = poisson_requests(seed=5, rate=20.0, duration=30.0)
    assert [(r.arrival, r.radius, r.levels, r.re, r.oscillating) for r in a] == \
           [(r.arrival, r.radius, r.levels, r.re, r.oscillating) for r in b]
    assert 450 < len(a) < 750                       # 20/s over 30 s
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0) and arr[-1] <= 30.0
    assert all(3.0 <= r.radius <= 8.0 and 1 <= r.levels <= 3 and 20.0 <= r.re <= 300.0 for r in a)
    osc = np.mean([r.oscillating for r in a])
    assert 0.4 < osc < 0.6
    gaps = np.diff(np.concatenate([[0.0], arr]))
    assert abs(gaps.mean() - 1 / 20.0) < 0.01


def test_request_case_on_template():
    from mortontrie_amr_b200.serving import (U_INLET, Request, build_template, footprint_bytes, request_case,
                                             template_key)
    req = Request(rid=0, arrival=0.0, radius=3.4, levels=2, re=150.0, oscillating=True)
    assert template_key(req) == (4, 2, True)
    mesh = build_template(template_key(req))
    case = request_case(req, mesh)
    s = 1 << req.levels
    r = np.linalg.norm(case.mesh.markers.ref, axis=0)
    assert np.allclose(r, req.radius * s)
    assert abs(case.mesh.markers.dv.sum() - 4 * np.pi * (req.radius * s) ** 2) < 1e-6
    # the oscillation path: amplitude R/2 along y, one period of 2000 finest steps
    p = case.mesh.markers.path
    assert p.shape == (2000, 6) and abs(p[:, 1].max() - 0.5 * req.radius * s) < 1e-3
    assert np.isclose(case.params.nu, U_INLET * 2 * req.radius / req.re)
    assert case.mesh.levels[2]["lat_f"] is mesh.levels[2]["lat_f"]   # shared host mesh
    assert footprint_bytes(case, "f16") < footprint_bytes(case, "f64")
    # every stencil cell of every marker over the path lies in the forcing band
    from mortontrie_amr_b200.lattice import cell_coords
    bx, by, bz = cell_coords(2, 2, mesh.levels[2]["ib_band"])
    band = set(zip(bx.tolist(), by.tolist(), bz.tolist()))
    c = np.array(case.mesh.markers.center)
    for t in (0, 500, 1000, 1500):
        pos = c[:, None] + p[t, :3, None] + case.mesh.markers.ref
        base = np.floor(pos).astype(int)
        for d in np.ndindex(3, 3, 3):
            cells = base + (np.array(d) - 1)[:, None]
            assert all(tuple(x) in band for x in cells.T[::37])


def test_device_template_request_case():
    """With device meshes a request's case is a spec fitted to its own radius
    and amplitude (band slack 0) on the template's boxes."""
    from mortontrie_amr_b200.mesh import SpecMesh
    from mortontrie_amr_b200.serving import Request, TemplateCache, footprint_bytes, request_case
    req = Request(rid=0, arrival=0.0, radius=3.4, levels=2, re=150.0, oscillating=True)
    cache = TemplateCache()
    tmpl = cache.get(req)
    assert isinstance(tmpl, SpecMesh) and tmpl.spec.sphere.radius == 4.0
    case = request_case(req, tmpl)
    assert isinstance(case.mesh, SpecMesh)
    sp = case.mesh.spec
    assert sp.sphere.radius == 3.4 and sp.band_slack == 0.0 and sp.oscillation == (0.5 * 3.4, 2000)
    assert sp.refine == tmpl.spec.refine
    assert np.allclose(np.linalg.norm(case.mesh.markers.ref, axis=0), 3.4 * 4)
    assert footprint_bytes(case, "f16") < footprint_bytes(case, "f64")


def test_estimated_cells_bound_the_host_mesh():
    from mortontrie_amr_b200.case import cavity_case, df_sphere_case, nested_sphere_case, sphere_case
    from mortontrie_amr_b200.mesh import estimate_cells
    for case in (sphere_case(), df_sphere_case(radius=3, max_level=2, oscillating=True),
                 cavity_case(coarse=(24, 24, 24), max_level=2),
                 nested_sphere_case(coarse=(48, 24, 24), max_level=2, center=(16, 12, 12), radius=2.0,
                                    half_widths=(4.0, 2.5))):
        est = estimate_cells(case.mesh.spec)
        got = case.mesh.n_cells()
        assert all(e >= g for e, g in zip(est, got)), (est, got)
        assert sum(est) <= 1.3 * sum(got), (est, got)


def test_summary_counts_finite_results_only():
    """cases/h, p50 and p99 of the request loop count finite results; a
    request whose state diverged (guard) or whose drag is NaN is failed."""
    from mortontrie_amr_b200.serving import Result, ServerStats
    rs = [Result(rid=0, arrival=0, admitted=0, finished=1, cd=1.0, cl=0, coarse_steps=1, storage="f16"),
          Result(rid=1, arrival=0, admitted=0, finished=2, cd=1.0, cl=0, coarse_steps=1, storage="f16",
                 finite=False),
          Result(rid=2, arrival=0, admitted=0, finished=9, cd=float("nan"), cl=0, coarse_steps=1, storage="f16")]
    s = ServerStats(results=rs, wall_s=3600.0).summary()
    assert s["completed"] == 3 and s["finite"] == 1 and s["failed"] == 2
    assert s["cases_per_hour"] == 1.0 and s["p99_s"] == 1.0


def test_octree_templates():
    """Templates refined from the forcing band (refine="octree"): the host
    template's band equals the box template's, with fewer cells; a request
    on a device template keeps the octree and takes its own radius and path."""
    from mortontrie_amr_b200.mesh import SpecMesh, estimate_cells
    from mortontrie_amr_b200.serving import Request, TemplateCache, build_template, request_case
    key = (3, 2, True)
    box = build_template(key, "host")
    oc = build_template(key, "host", refine="octree")
    assert np.array_equal(oc.levels[2]["ib_band"], box.levels[2]["ib_band"])
    assert sum(oc.n_cells()) < sum(box.n_cells())
    req = Request(rid=0, arrival=0.0, radius=2.6, levels=2, re=80.0, oscillating=True, finest_steps=2000)
    case = request_case(req, TemplateCache(refine="octree").get(req))
    assert isinstance(case.mesh, SpecMesh) and case.mesh.spec.octree is not None
    assert case.mesh.spec.sphere.radius == 2.6
    est = estimate_cells(case.mesh.spec)
    assert est[2] < estimate_cells(request_case(req, TemplateCache().get(req)).mesh.spec)[2]
