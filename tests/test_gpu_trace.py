"""The FP64 GPU path against the reference's own multi-dump traces, through
the C ABI, under the reference's phase order and under the fused schedule:

* cfg1 (64x32x32 coarse, 2 levels, sphere R = 4, Re 20) for 1000 coarse
  steps, closed by the non-equilibrium boundary on every face, and with
  periodic y / z sides;
* four levels: the D3Q27 cumulant sphere scaled to 48x24x24 coarse (20
  coarse = 160 finest steps) and a D3Q19 distance-weighted sphere.

Bit-exact populations (f on every non-boundary cell, fcol everywhere),
rho and u on lat_f after every recorded step count; the IB force summed up
to each count within 1e-12 (the reference sums it in map order)."""
import numpy as np
import pytest
from golden_cases import TRACE_CASES
from helpers import init_of, load_trace, rel_err, trace_mismatches

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from mortontrie_amr_b200.lbm import Context
    c = Context(0)
    yield c
    c.close()


def gpu_state(mgr):
    def get(l):
        keys, tags = mgr.keys(l)
        f, fcol = mgr.populations(l)
        rho, u = mgr.macros(l)
        return dict(keys=keys, tags=tags, f=f, fcol=fcol, rho=rho, u=u)
    return get


@pytest.mark.parametrize("schedule", ["phases", "fused"])
@pytest.mark.parametrize("name", sorted(TRACE_CASES))
def test_gpu_matches_reference_trace(ctx, name, schedule):
    from mortontrie_amr_b200.lbm import LBM_Manager
    spec, case, z, _ = load_trace(name)
    mgr = LBM_Manager(ctx, case, schedule=schedule)
    init = init_of(case, spec)
    if init is not None:
        for l, (keys, f) in enumerate(init):
            mgr.set_populations(l, f)
    done = 0
    for d, n in enumerate(spec["dumps"]):
        mgr.fluidSimulate(n - done)
        done = n
        ctx.synchronize()
        bad = trace_mismatches(case, z, d, gpu_state(mgr))
        assert bad == [], (name, schedule, n, bad)
        force = mgr.force()
        ref = z["force"][:n].sum(axis=0)
        assert force[3] == ref[3]
        if np.abs(ref[:3]).max() > 0:
            assert rel_err(force[:3], ref[:3]) < 1e-12, (name, schedule, n)
    mgr.close()
