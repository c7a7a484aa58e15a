"""The request loop on the device: requests arriving while others run join
the batch (continuous batching), and each result is the same as the request
solved alone, within the stated tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# drag and lift of a request in the mix vs alone (FP16 storage, same kernels
# but batched: identical arithmetic up to FMA contraction in the batched pass)
TOL_MIX = 1e-5


@pytest.fixture(scope="module")
def ctx():
    from mortontrie_amr_b200.lbm import Context
    c = Context(0)
    yield c
    c.close()


def _stream():
    from mortontrie_amr_b200.serving import Request
    spec = [(0.00, 3.0, 1, 60.0, True), (0.00, 3.6, 2, 120.0, False), (0.02, 4.0, 1, 200.0, True),
            (0.05, 3.2, 2, 40.0, True), (0.10, 3.9, 1, 90.0, False), (0.15, 3.5, 2, 250.0, True)]
    return [Request(rid=i, arrival=a, radius=r, levels=l, re=re, oscillating=o, finest_steps=96)
            for i, (a, r, l, re, o) in enumerate(spec)]


def test_served_results_equal_alone(ctx):
    from mortontrie_amr_b200.serving import Server, TemplateCache, solve_alone
    reqs = _stream()
    cache = TemplateCache()
    cache.prepare(reqs)
    server = Server(ctx, cache, storage="f16", chunk=4)
    stats = server.run(reqs, realtime=True)
    assert len(stats.results) == len(reqs)
    assert stats.max_resident >= 2              # requests overlapped on the device
    by_id = {r.rid: r for r in stats.results}
    for req in reqs:
        cd, cl, _ = solve_alone(ctx, cache, req, storage="f16")
        r = by_id[req.rid]
        assert np.isfinite(r.cd) and abs(r.cd - cd) <= TOL_MIX * max(abs(cd), 1e-3), (req, r.cd, cd)
        assert abs(r.cl - cl) <= TOL_MIX * max(abs(cd), 1e-3), (req, r.cl, cl)
        assert r.finished >= r.admitted >= r.arrival - 1e-9


def test_budget_limits_residency(ctx):
    """With a budget below two cases, requests run one at a time."""
    from mortontrie_amr_b200.serving import Server, TemplateCache, footprint_bytes, request_case
    reqs = _stream()[:3]
    cache = TemplateCache()
    cache.prepare(reqs)
    small = min(footprint_bytes(request_case(r, cache.get(r)), "f16") for r in reqs)
    server = Server(ctx, cache, storage="f16", budget_gb=1.5 * small / 1e9, chunk=4)
    stats = server.run(reqs, realtime=False)
    assert len(stats.results) == 3 and stats.max_resident == 1


def test_markers_and_async_force(ctx):
    """A marker recorded after queued steps turns done once the stream passes
    it, without synchronising; the force copied asynchronously before it
    equals the synchronous read; tickets older than the marker ring read as
    done."""
    import time
    from mortontrie_amr_b200.serving import Request, TemplateCache, request_case
    from mortontrie_amr_b200.lbm import LBM_Manager
    req = Request(rid=0, arrival=0.0, radius=3.3, levels=2, re=80.0, oscillating=True, finest_steps=64)
    mgr = LBM_Manager(ctx, request_case(req, TemplateCache().get(req)), "f16", schedule="fused")
    first = ctx.marker()
    mgr.fluidSimulate(16)
    mgr.force_async()
    tk = ctx.marker()
    assert tk > first
    t0 = time.time()
    while not ctx.marker_done(tk):
        assert time.time() - t0 < 60.0
        time.sleep(0.001)
    assert np.array_equal(mgr.force_copied(), mgr.force())
    assert mgr.force()[3] > 0
    for _ in range(70):
        ctx.marker()
    assert ctx.marker_done(first)
    mgr.close()


def test_async_guard_flags_nonfinite_state(ctx):
    """The guard enqueued with the force copy: a healthy state reads finite;
    a state given a NaN population on the host (the failure is made on the
    host, no kernel is driven into a fault) reads non-finite under the next
    marker."""
    import time
    from mortontrie_amr_b200.lbm import LBM_Manager
    from mortontrie_amr_b200.serving import Request, TemplateCache, request_case
    req = Request(rid=0, arrival=0.0, radius=3.3, levels=1, re=80.0, oscillating=False, finest_steps=32)
    mgr = LBM_Manager(ctx, request_case(req, TemplateCache().get(req)), "f16", schedule="fused")

    def guard_after_marker():
        mgr.force_async()
        tk = ctx.marker()
        t0 = time.time()
        while not ctx.marker_done(tk):
            assert time.time() - t0 < 60.0
            time.sleep(0.001)
        return mgr.finite_copied()

    mgr.fluidSimulate(4)
    assert guard_after_marker()
    f, fcol = mgr.populations(1)
    fcol[5, fcol.shape[1] // 2] = np.nan
    mgr.set_populations(1, f, fcol)
    assert not guard_after_marker()
    mgr.close()
