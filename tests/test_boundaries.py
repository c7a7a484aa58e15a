"""Restated domain boundaries on the CPU oracle (no runnable reference code:
BC/ZouHe_Velocity.cpp and BC/Outflow.cpp need the ghost layers that
BC_NO_GHOST removes; parity with the reference is unpinned for them).  The
Zou-He / Hecht-Harting velocity inlet with the five-population outflow
(bc_mode "zouhe_hh") drives an empty periodic channel started at rest to the
inlet velocity, under both stream directions."""
import numpy as np
import pytest


def _channel(conv, n=(32, 8, 8), u=0.05):
    from mortontrie_amr_b200.case import Case, CaseParams
    from mortontrie_amr_b200.mesh import MeshSpec, build_mesh
    spec = MeshSpec(q=19, max_level=1, coarse=n, refine=[None], boundary=("bc", "periodic", "periodic"))
    p = CaseParams(q=19, collision="LBGK", ib_method="FH", bc_mode="zouhe_hh", nu=0.05, u_bc=(u, 0.0, 0.0),
                   u_ref=u, stream_convention=conv)
    return Case(build_mesh(spec), p)


@pytest.mark.parametrize("conv", ["reference", "textbook"])
def test_hh_inlet_drives_channel_to_inlet_velocity(conv):
    import oracle as O
    from mortontrie_amr_b200.case import equilibrium
    from mortontrie_amr_b200.lattice import cell_coords
    case = _channel(conv)
    oc = O.OracleCase(case)
    n = oc.size(0)
    oc.set_populations(0, equilibrium(19, np.ones(n), np.zeros(n), np.zeros(n), np.zeros(n)))
    oc.step(400)
    g = oc.get(0)
    x, _, _ = cell_coords(1, 0, g["keys"])
    fluid = (g["tags"] & 1) > 0
    assert np.isfinite(g["f"]).all()
    for xx in (1, 8, 16, 24, 30):
        ux = g["u"][fluid & (x == xx), 0]
        assert np.allclose(ux, 0.05, rtol=0.03), (conv, xx, ux.min(), ux.max())
    assert np.abs(g["u"][fluid, 1:]).max() < 1e-10          # no transverse flow in a plug


def test_hh_mode_is_d3q19_lbgk():
    import oracle as O
    from mortontrie_amr_b200.case import Case, CaseParams
    from mortontrie_amr_b200.mesh import MeshSpec, build_mesh
    spec = MeshSpec(q=27, max_level=1, coarse=(8, 8, 8), refine=[None], boundary=("bc", "periodic", "periodic"))
    p = CaseParams(q=27, collision="Cumulant", bc_mode="zouhe_hh", u_bc=(0.05, 0, 0), u_ref=0.05)
    with pytest.raises(ValueError):
        O.OracleCase(Case(build_mesh(spec), p))
