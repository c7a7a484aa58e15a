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
    from mortontrie_amr_b200.serving import Request, build_template, footprint_bytes, request_case, template_key
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
    assert np.isclose(case.params.nu, 0.05 * 2 * req.radius / req.re)
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
