"""Specifications of the cases whose reference outputs are stored as golden
vectors.  Shared by gen_golden.py and the tests, so both rebuild the same
index sets with the mesher."""
from __future__ import annotations

import numpy as np

from mortontrie_amr_b200.case import Case, CaseParams
from mortontrie_amr_b200.mesh import MeshSpec, Sphere, build_mesh

GOLDEN_CASES = {
    # single populated level in a non-equilibrium-extrapolation box (LBGK Q19)
    "box_q19_neq": dict(q=19, collision="LBGK", coarse=(10, 8, 8), max_level=1, refine=[None], sphere=None,
                        boundary=("bc", "bc", "bc"), nu=0.02, u=0.05, ib="FH", steps=6, seed=7, init="perturbed"),
    # two levels with a sphere: explosion, coalescence, Filippova-Haenel links, clamp, MDF
    "sphere_q19_fh": dict(q=19, collision="LBGK", coarse=(16, 12, 12), max_level=1, refine=[((4, 3, 3), (12, 9, 9))],
                          sphere=((8.0, 6.0, 6.0), 1.4), boundary=("bc", "bc", "bc"), nu=0.015, u=0.05, ib="FH",
                          steps=4, seed=11, init="perturbed"),
    # the same from the reference's own initial state (f = feq(rho0, u_bc))
    "sphere_q19_fh_refinit": dict(q=19, collision="LBGK", coarse=(16, 12, 12), max_level=1,
                                  refine=[((4, 3, 3), (12, 9, 9))], sphere=((8.0, 6.0, 6.0), 1.4),
                                  boundary=("bc", "bc", "bc"), nu=0.015, u=0.05, ib="FH", steps=5, seed=0,
                                  init="reference"),
    # D3Q27 cumulant across a refinement interface
    "refined_q27_cumulant": dict(q=27, collision="Cumulant", coarse=(12, 10, 10), max_level=1,
                                 refine=[((3, 3, 3), (9, 7, 7))], sphere=None, boundary=("bc", "bc", "bc"), nu=0.01,
                                 u=0.04, ib="FH", steps=4, seed=5, init="perturbed"),
    # three levels, distance-weighted links
    "sphere_q19_dw_l2": dict(q=19, collision="LBGK", coarse=(14, 12, 12), max_level=2,
                             refine=[((4, 3, 3), (10, 9, 9)), ((11, 9, 9), (17, 15, 15))],
                             sphere=((7.0, 6.0, 6.0), 0.6), boundary=("bc", "bc", "bc"), nu=0.005, u=0.05, ib="DW",
                             steps=2, seed=3, init="perturbed"),
}

# Runs whose reference state is recorded after several coarse-step counts
# ("dumps"): SHA-256 of every level's arrays, a sample of cells in full, and
# the per-step IB force series (gen_golden.py --trace).
TRACE_CASES = {
    # cfg1 geometry (64x32x32 coarse, 2 levels, refined box (4,8,8)-(28,24,24),
    # sphere R = 4 at (16,16,16), Re 20: nu = 0.05 * 8 / 20), closed by the
    # reference's live non-equilibrium boundary on every face, from the
    # reference's own initial state, 1000 coarse steps
    "cfg1_neq_1000": dict(q=19, collision="LBGK", coarse=(64, 32, 32), max_level=1, refine=[((4, 8, 8), (28, 24, 24))],
                          sphere=((16.0, 16.0, 16.0), 4.0), boundary=("bc", "bc", "bc"), nu=0.02, u=0.05, ib="FH",
                          seed=0, init="reference", dumps=[10, 100, 1000]),
    # the same with periodic y and z (the cfg1 lateral sides), non-equilibrium
    # boundary on the West and East faces
    "cfg1_periodic_1000": dict(q=19, collision="LBGK", coarse=(64, 32, 32), max_level=1,
                               refine=[((4, 8, 8), (28, 24, 24))], sphere=((16.0, 16.0, 16.0), 4.0),
                               boundary=("bc", "periodic", "periodic"), nu=0.02, u=0.05, ib="FH", seed=0,
                               init="reference", dumps=[10, 100, 1000]),
    # the 4-level D3Q27 cumulant sphere scaled by 1/4 (48x24x24 coarse, R = 1.5
    # coarse = 12 finest cells, nested half-widths 4R, 2.5R, 1.75R, Re 200,
    # u 0.04), 12 coarse steps = 96 finest steps (the reference itself turns
    # non-finite between coarse steps 14 and 15 of this case)
    "cfg3_small_q27_l3": dict(q=27, collision="Cumulant", coarse=(48, 24, 24), max_level=3,
                              refine=[((10, 6, 6), (22, 18, 18)), ((24, 16, 16), (40, 32, 32)),
                                      ((54, 38, 38), (74, 58, 58))],
                              sphere=((16.0, 12.0, 12.0), 1.5), boundary=("bc", "bc", "bc"), nu=0.0006, u=0.04,
                              ib="FH", seed=0, init="reference", dumps=[2, 12]),
    # four levels of D3Q19 LBGK with distance-weighted links from a perturbed state
    "nested_q19_dw_l3": dict(q=19, collision="LBGK", coarse=(28, 16, 16), max_level=3,
                             refine=[((4, 2, 2), (16, 14, 14)), ((13, 9, 9), (27, 23, 23)),
                                     ((32, 24, 24), (48, 40, 40))],
                             sphere=((10.0, 8.0, 8.0), 1.0), boundary=("bc", "bc", "bc"), nu=0.002, u=0.05, ib="DW",
                             seed=21, init="perturbed", dumps=[1, 6]),
}


def build_case(spec) -> Case:
    sphere = Sphere(tuple(spec["sphere"][0]), spec["sphere"][1]) if spec["sphere"] else None
    refine = [None if r is None else (tuple(r[0]), tuple(r[1])) for r in spec["refine"]]
    ms = MeshSpec(q=spec["q"], max_level=spec["max_level"], coarse=tuple(spec["coarse"]), refine=refine,
                  boundary=tuple(spec["boundary"]), sphere=sphere)
    p = CaseParams(q=spec["q"], collision=spec["collision"], ib_method=spec["ib"], bc_mode="neq", nu=spec["nu"],
                   u_bc=(spec["u"], 0.0, 0.0), u_ref=spec["u"])
    return Case(build_mesh(ms), p)


def dis_mesh(spec):
    """The two-level STL sphere mesh of a wall-distance golden and its
    triangles (coarse units)."""
    from mortontrie_amr_b200.stl import icosphere
    tris = icosphere(spec["center"], spec["radius"], spec["sub"])
    mesh = build_mesh(MeshSpec(q=spec["q"], max_level=1, coarse=(32, 16, 16), refine=[((6, 4, 4), (18, 12, 12))],
                               boundary=("bc", "periodic", "periodic"), surface=tris))
    return mesh, tris


# single-cell collision known answers: a closed 10^3 box (its 8^3 interior
# collides), one coarse step of the reference's own code from seeded random
# cell states; the fixture keeps SAMPLE_CELLS interior cells' inputs and
# post-collision outputs
COLLIDE_CASES = {
    "collide_q19_lbgk": dict(q=19, collision="LBGK", nu=0.02),
    "collide_q27_cumulant": dict(q=27, collision="Cumulant", nu=0.005),
    "collide_q27_lbgk": dict(q=27, collision="LBGK", nu=0.01),
}
COLLIDE_SEED = 1234
SAMPLE_CELLS = 64


def collide_case(spec):
    from mortontrie_amr_b200.case import uniform_box_case
    return uniform_box_case(q=spec["q"], n=(10, 10, 10), nu=spec["nu"], boundary=("bc", "bc", "bc"),
                            collision=spec["collision"], empty_levels=1)


def collide_state(case, seed=COLLIDE_SEED):
    """Seeded per-cell states of every level-0 cell: rho in U[0.9, 1.1), u of
    uniform direction and |u| in U[0, 0.1), the BGK equilibrium of those
    plus a non-equilibrium part 0.01 w_q N(0, 1).  Returns the harness's
    init list (level 0 keys and f; the empty level 1)."""
    from mortontrie_amr_b200.case import equilibrium
    from mortontrie_amr_b200.lattice import weights
    q = case.params.q
    keys = case.mesh.all_keys(0)
    rng = np.random.default_rng(seed)
    n = keys.size
    rho = rng.uniform(0.9, 1.1, n)
    d = rng.standard_normal((3, n))
    d /= np.linalg.norm(d, axis=0)
    u = d * rng.uniform(0.0, 0.1, n)
    f = equilibrium(q, rho, u[0], u[1], u[2]) + 0.01 * weights(q)[:, None] * rng.standard_normal((q, n))
    return [(keys, f), (case.mesh.all_keys(1), np.zeros((q, 0)))]


def collide_sample(case, seed=COLLIDE_SEED):
    """Indices (into the level-0 keys) of the sampled interior cells."""
    lat_f = case.mesh.levels[0]["lat_f"]
    keys = case.mesh.all_keys(0)
    idx = np.searchsorted(keys, lat_f)
    rng = np.random.default_rng(seed + 1)
    return np.sort(rng.choice(idx, size=SAMPLE_CELLS, replace=False))


# the uniform periodic Taylor-Green configuration (the dense path's
# workload), small enough for the reference's own code
TGV_CASES = {
    "tgv_q19_32_periodic": dict(q=19, collision="LBGK", n=32, steps=10, nu=1.0 / 30.0, u0=0.02),
    "tgv_q27_cumulant_16_periodic": dict(q=27, collision="Cumulant", n=16, steps=10, nu=1.0 / 30.0, u0=0.02),
    "tgv_q27_lbgk_16_periodic": dict(q=27, collision="LBGK", n=16, steps=10, nu=1.0 / 30.0, u0=0.02),
}


def tgv_fields(spec):
    from mortontrie_amr_b200.case import taylor_green_fields
    from mortontrie_amr_b200.lbm import morton_order_fields
    n = spec["n"]
    return morton_order_fields(n, *taylor_green_fields((n, n, n), spec["u0"]))


def tgv_reference_case(spec):
    """The case as the reference harness runs it (an empty second level, the
    periodic wrap) and its initial state: the BGK equilibrium of the fields."""
    from mortontrie_amr_b200.case import equilibrium, uniform_box_case
    n, q = spec["n"], spec["q"]
    case = uniform_box_case(q=q, n=(n, n, n), nu=spec["nu"], boundary=("periodic",) * 3, empty_levels=1,
                            u_ref=spec["u0"], collision=spec["collision"])
    f0 = equilibrium(q, *tgv_fields(spec))
    return case, [(case.mesh.all_keys(0), f0), (case.mesh.all_keys(1), np.zeros((q, 0)))]
