"""Python host mirror of the reference's LBM call surface over the C ABI.

The class and method names follow the reference's interface
(header/LBM_Manager.hpp:25-119, header/lbm_kernel/Collision_Manager.hpp:73-97,
header/lbm_kernel/Stream_Manager.hpp:12-37, header/ComplexBoundary_Manager.hpp
:16-46, header/BC/D3Q19_BC_Manager.hpp:201-263); every call goes through
libmtlbm.so (include/mt_lbm.h).  There is no CPU fallback: importing this
module raises if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .case import BC_MODES, COLLISIONS, IB_METHODS, STORAGE, STREAM_CONVENTIONS, Case
from .mesh import SpecMesh

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmtlbm.so")

MAX_LEVELS = 8
SET_IDS = {"lat_f": 0, "overlap_F2C": 1, "overlap_C2F": 2, "ghost_overlap_C2F": 3, "ghost_overlap_F2C": 4,
           "lat_sf": 5, "ib_band": 6}
SET_LAT_BC0 = 16
ERRORS = {-1: "MT_ERR_ARG", -2: "MT_ERR_CUDA", -3: "MT_ERR_STATE", -4: "MT_ERR_MESH", -5: "MT_ERR_NONFINITE"}
EXPORTS = [
    "mt_create", "mt_destroy", "mt_last_error", "mt_set_stream", "mt_synchronize", "mt_launch_count",
    "mt_case_create", "mt_case_create_dense", "mt_case_destroy", "mt_case_add_set", "mt_case_set_dis",
    "mt_case_build", "mt_case_level_size", "mt_case_get_keys", "mt_case_get_neighbors", "mt_find",
    "mt_case_init_equilibrium", "mt_case_init_fields", "mt_case_set_populations", "mt_case_get_populations",
    "mt_case_get_macros", "mt_case_reduce", "mt_calculate_macros", "mt_collide", "mt_stream", "mt_explosion",
    "mt_coalescence", "mt_apply_bc", "mt_apply_bc_face", "mt_ib_treat", "mt_lbm_kernel", "mt_step", "mt_get_force",
    "mt_reset_force", "mt_case_tune", "mt_case_status", "mt_case_reduce_noalloc", "mt_case_reduce_levels", "mt_case_info", "mt_case_get_step", "mt_case_set_step",
    "mt_case_get_df_force_field", "mt_case_set_df_force_field", "mt_case_set_schedule", "mt_case_set_interface_scaling", "mt_case_set_interface_time", "mt_case_set_face_velocity", "mt_case_set_markers",
    "mt_batch_create", "mt_batch_destroy", "mt_batch_add", "mt_batch_remove", "mt_batch_size", "mt_batch_step", "mt_case_prepare", "mt_case_transfer",
    "mt_case_generate", "mt_case_set_surface", "mt_case_set_region", "mt_marker_record", "mt_marker_done", "mt_case_force_async",
    "mt_case_force_copied", "mt_set_priority", "mt_case_remap", "mt_case_status_copied", "mt_case_tune_bricks",
    "mt_case_set_brick_forms",
]


SCHEDULES = {"phases": 0, "fused": 1, "fused_lists": 2}
SCALINGS = {"reference": 0, "standard": 1}
ITIMES = {"reference": 0, "hold": 1, "extrap": 2}
BRICK_FORMS = 4  # MT_BRICK_FORMS


class MTError(RuntimeError):
    pass


class mt_case_desc(C.Structure):
    _fields_ = [("q", C.c_int32), ("max_level", C.c_int32), ("collision", C.c_int32), ("ib_method", C.c_int32),
                ("bc_mode", C.c_int32), ("stream_convention", C.c_int32), ("storage", C.c_int32),
                ("periodic", C.c_int32 * 3), ("extent0", C.c_int64 * 3), ("tau", C.c_double * MAX_LEVELS),
                ("rho0", C.c_double), ("u_bc", C.c_double * 3),
                ("u_shift", (C.c_double * 3) * MAX_LEVELS)]


class mt_mesh_spec(C.Structure):
    _fields_ = [("coarse", C.c_int64 * 3), ("boundary_bc", C.c_int32 * 3), ("has_refine", C.c_int32 * MAX_LEVELS),
                ("refine_lo", (C.c_int64 * 3) * MAX_LEVELS), ("refine_hi", (C.c_int64 * 3) * MAX_LEVELS),
                ("sphere", C.c_int32), ("pad", C.c_int32), ("center", C.c_double * 3), ("radius", C.c_double),
                ("osc_amplitude", C.c_double), ("band_slack", C.c_double)]


def make_mesh_spec(spec) -> mt_mesh_spec:
    """mt_mesh_spec of a MeshSpec (mesh.py): the device classification
    produces the sets build_mesh(spec) would.  An octree's levels are marked
    as regions (has_refine 2), uploaded by upload_regions."""
    octree = getattr(spec, "octree", None) is not None
    if not octree and len(spec.refine) != spec.max_level:
        raise ValueError("need one refinement box per level below the maximum level")
    if spec.max_level >= MAX_LEVELS:
        raise ValueError("too many levels")
    m = mt_mesh_spec()
    for a in range(3):
        m.coarse[a] = int(spec.coarse[a])
        m.boundary_bc[a] = int(spec.boundary[a] == "bc")
    if octree:
        for l in range(spec.max_level):
            m.has_refine[l] = 2
    for l, box in enumerate([] if octree else spec.refine):
        if box is None:
            break
        m.has_refine[l] = 1
        for a in range(3):
            m.refine_lo[l][a] = int(box[0][a])
            m.refine_hi[l][a] = int(box[1][a])
    if getattr(spec, "surface", None) is not None:
        m.sphere = 3
    elif spec.sphere is not None:
        m.sphere = 2 if spec.ib == "markers" else 1
        for a in range(3):
            m.center[a] = float(spec.sphere.center[a])
        m.radius = float(spec.sphere.radius)
        m.osc_amplitude = float(spec.oscillation[0]) if (spec.ib == "markers" and spec.oscillation) else 0.0
        m.band_slack = float(spec.band_slack)
    return m


def _storage_code(storage) -> int:
    from .case import STORAGE
    return STORAGE[storage]


def upload_regions(ctx, case_id, spec):
    """The octree's refinement regions (mesh.octree_regions, made on the
    host) for mt_case_generate, each cropped to the box of its cells."""
    from .mesh import octree_regions
    regions = octree_regions(spec)
    for l in range(1, spec.max_level + 1):
        r = regions[l]
        ix, iy, iz = np.nonzero(r.mask)
        lo = np.array([ix.min(), iy.min(), iz.min()], np.int64)
        hi = np.array([ix.max(), iy.max(), iz.max()], np.int64) + 1
        mask = np.ascontiguousarray(r.mask[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]], np.uint8)
        blo = np.ascontiguousarray(lo + r.lo, np.int64)
        shape = np.ascontiguousarray(hi - lo, np.int64)
        ctx.check(lib().mt_case_set_region(ctx.h, case_id, l, _ptr(blo, C.c_int64), _ptr(shape, C.c_int64),
                                           _ptr(mask, C.c_uint8)), "mt_case_set_region")


_lib = None


def lib():
    """Load libmtlbm.so; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MTError(f"{LIB_PATH} is missing: run mortontrie_amr_b200/build.py (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
        u64p, i64p, i32p, u32p, dp = (C.POINTER(C.c_uint64), C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                      C.POINTER(C.c_uint32), C.POINTER(C.c_double))
        sig = {
            "mt_create": [i32, C.POINTER(vp)], "mt_destroy": [vp], "mt_set_stream": [vp, vp], "mt_synchronize": [vp],
            "mt_launch_count": [vp, i64p], "mt_case_create": [vp, C.POINTER(mt_case_desc), i32p],
            "mt_case_create_dense": [vp, C.POINTER(mt_case_desc), i32p], "mt_case_destroy": [vp, i32],
            "mt_case_add_set": [vp, i32, i32, i32, u64p, i64], "mt_case_set_dis": [vp, i32, u64p, dp, i64],
            "mt_case_build": [vp, i32], "mt_case_level_size": [vp, i32, i32, i64p],
            "mt_case_get_keys": [vp, i32, i32, u64p, u32p], "mt_case_get_neighbors": [vp, i32, i32, i32p],
            "mt_find": [vp, i32, i32, u64p, i64, i64p], "mt_case_init_equilibrium": [vp, i32, C.c_double, dp],
            "mt_case_init_fields": [vp, i32, dp, dp, dp, dp], "mt_case_set_populations": [vp, i32, i32, dp, dp],
            "mt_case_get_populations": [vp, i32, i32, dp, dp], "mt_case_get_macros": [vp, i32, i32, dp, dp],
            "mt_case_reduce": [vp, i32, dp], "mt_case_reduce_noalloc": [vp, i32, dp], "mt_case_reduce_levels": [vp, i32, dp], "mt_case_info": [vp, i32, dp], "mt_case_get_step": [vp, i32, i64p], "mt_case_set_step": [vp, i32, i64],
            "mt_case_get_df_force_field": [vp, i32, i64p], "mt_case_set_df_force_field": [vp, i32, i64p], "mt_case_set_schedule": [vp, i32, i32], "mt_case_set_interface_scaling": [vp, i32, i32], "mt_case_set_interface_time": [vp, i32, i32], "mt_case_set_face_velocity": [vp, i32, i32, dp], "mt_case_set_markers": [vp, i32, i64, dp, dp, dp, i64, dp],
            "mt_batch_create": [vp, i32p], "mt_batch_destroy": [vp, i32], "mt_batch_add": [vp, i32, i32],
            "mt_batch_remove": [vp, i32, i32], "mt_batch_size": [vp, i32, i32p], "mt_batch_step": [vp, i32, i32], "mt_case_prepare": [vp, i32], "mt_case_transfer": [vp, i32, vp, i32p],
            "mt_case_generate": [vp, i32, C.POINTER(mt_mesh_spec)], "mt_case_set_surface": [vp, i32, dp, i64],
            "mt_case_set_region": [vp, i32, i32, i64p, i64p, C.POINTER(C.c_uint8)],
            "mt_marker_record": [vp, i64p], "mt_marker_done": [vp, i64, i32p], "mt_case_force_async": [vp, i32],
            "mt_case_force_copied": [vp, i32, dp], "mt_case_status_copied": [vp, i32], "mt_case_tune_bricks": [vp, i32, i32p, C.POINTER(C.c_float)], "mt_case_set_brick_forms": [vp, i32, i32p], "mt_set_priority": [vp, i32], "mt_case_remap": [vp, i32, i32, i64p], "mt_calculate_macros": [vp, i32, i32], "mt_collide": [vp, i32, i32],
            "mt_stream": [vp, i32, i32], "mt_explosion": [vp, i32, i32], "mt_coalescence": [vp, i32, i32],
            "mt_apply_bc": [vp, i32], "mt_apply_bc_face": [vp, i32, i32], "mt_ib_treat": [vp, i32], "mt_lbm_kernel": [vp, i32, i32],
            "mt_step": [vp, i32, i32], "mt_get_force": [vp, i32, dp], "mt_reset_force": [vp, i32],
            "mt_case_tune": [vp, i32, i32p, C.POINTER(C.c_float)], "mt_case_status": [vp, i32],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.mt_last_error.argtypes = [vp]
        L.mt_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def _ptr(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Context:
    """One device context (mt_create); owns every case created on it."""

    def __init__(self, device: int = 0):
        self.device = device
        self.h = C.c_void_p()
        rc = lib().mt_create(device, C.byref(self.h))
        if rc != 0:
            raise MTError(f"mt_create failed ({ERRORS.get(rc, rc)})")

    def check(self, rc, what=""):
        if rc != 0:
            msg = lib().mt_last_error(self.h).decode()
            raise MTError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")

    def set_stream(self, cuda_stream_handle):
        self.check(lib().mt_set_stream(self.h, C.c_void_p(cuda_stream_handle or 0)), "mt_set_stream")

    def synchronize(self):
        self.check(lib().mt_synchronize(self.h), "mt_synchronize")

    def set_priority(self, high: bool = True):
        """Highest (or lowest) scheduling priority for the context's own stream."""
        self.check(lib().mt_set_priority(self.h, int(bool(high))), "mt_set_priority")

    def marker(self) -> int:
        """Ticket of the current point of the context stream (mt_marker_record)."""
        t = C.c_int64()
        self.check(lib().mt_marker_record(self.h, C.byref(t)), "mt_marker_record")
        return t.value

    def marker_done(self, ticket: int) -> bool:
        """Whether the stream has passed the marker (never blocks)."""
        d = C.c_int32()
        self.check(lib().mt_marker_done(self.h, int(ticket), C.byref(d)), "mt_marker_done")
        return bool(d.value)

    def launch_count(self) -> int:
        v = C.c_int64()
        self.check(lib().mt_launch_count(self.h, C.byref(v)), "mt_launch_count")
        return v.value

    def close(self):
        if self.h:
            lib().mt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def storage_shift_of(case: Case, storage_shift) -> list:
    """The shift velocity u_s of the reduced storages per level (a list of
    max_level + 1 triples): None (f - w_q on every level), "inlet" (the
    case's boundary velocity u_bc on every level), "far_field" (u_bc on the
    levels below the finest, zero on the finest, which holds the body), one
    velocity for every level, or one velocity per level."""
    nl = case.mesh.spec.max_level + 1
    ubc = tuple(float(v) for v in case.params.u_bc)
    zero = (0.0, 0.0, 0.0)
    if storage_shift is None:
        return [zero] * nl
    if isinstance(storage_shift, str):
        if storage_shift == "inlet":
            return [ubc] * nl
        if storage_shift == "far_field":
            return [ubc] * (nl - 1) + [zero]
        raise ValueError(f"storage_shift: None, 'inlet', 'far_field' or velocities, not {storage_shift!r}")
    a = np.asarray(storage_shift, np.float64)
    if a.shape == (3,):
        return [tuple(a.tolist())] * nl
    if a.shape == (nl, 3):
        return [tuple(r) for r in a.tolist()]
    raise ValueError(f"storage_shift needs 3 or ({nl}, 3) components, not {a.shape}")


def make_desc(case: Case, storage: str = None, storage_shift=None) -> mt_case_desc:
    p = case.params
    m = case.mesh
    d = mt_case_desc()
    d.q = p.q
    d.max_level = m.spec.max_level
    d.collision = COLLISIONS[p.collision]
    d.ib_method = IB_METHODS[p.ib_method]
    d.bc_mode = BC_MODES[p.bc_mode]
    d.stream_convention = STREAM_CONVENTIONS[p.stream_convention]
    d.storage = STORAGE[storage or p.storage]
    for a in range(3):
        d.periodic[a] = int(m.spec.boundary[a] == "periodic")
        d.extent0[a] = int(m.spec.coarse[a])
        d.u_bc[a] = float(p.u_bc[a])
    for l, u in enumerate(storage_shift_of(case, storage_shift)):
        for a in range(3):
            d.u_shift[l][a] = u[a]
    for l, t in enumerate(p.taus(m.spec.max_level)):
        d.tau[l] = float(t)
    d.rho0 = float(p.rho0)
    return d


class LBM_Manager:
    """Multi-level case on the device: the reference's LBM_Manager with its
    strategy objects (collide / stream / treat / boundary) as methods."""

    def __init__(self, ctx: Context, case: Case, storage: str = "f64", schedule: str = "phases",
                 scaling: str = "reference", generate: bool = False, storage_shift=None,
                 interface_time: str = "reference"):
        """storage: "f64" (the reference's precision, bit-exact) or "f32" /
        "f16" / "bf16" (FP32 arithmetic on stored deviations f - s_q).
        storage_shift: s_q = feq_q(1, u_s) of the reduced storages, per
        level; None (u_s = 0, s_q = w_q), "inlet" (u_s = the case's u_bc),
        "far_field" (u_bc below the finest level, 0 on it) or velocities
        (see storage_shift_of).
        schedule: "phases" (the reference's passes) or "fused" (stream fused
        with the next collision; same state after every coarse step).
        interface_time: "reference" (a fine level explodes in its first
        substep), "hold" (in both, from the parent's state of the step) or
        "extrap" (the second from that state extrapolated to the half step).
        generate: classify the lattice on the device from the mesh spec
        (mt_case_generate) instead of uploading the host mesher's sets; a
        SpecMesh (no host sets) is always generated."""
        self.ctx = ctx
        self.case = case
        self.q = case.params.q
        self.L = case.mesh.spec.max_level
        self.interface_time = interface_time
        self.storage = storage
        self.storage_shift = storage_shift_of(case, storage_shift)
        d = make_desc(case, storage, storage_shift)
        cid = C.c_int32()
        ctx.check(lib().mt_case_create(ctx.h, C.byref(d), C.byref(cid)), "mt_case_create")
        self.id = cid.value
        m = case.mesh
        if generate or isinstance(m, SpecMesh):
            ms = make_mesh_spec(m.spec)
            if getattr(m.spec, "octree", None) is not None:
                upload_regions(ctx, self.id, m.spec)
            if ms.sphere == 3:
                t = np.ascontiguousarray(m.spec.surface, np.float64).reshape(-1, 9)
                ctx.check(lib().mt_case_set_surface(ctx.h, self.id, _ptr(t, C.c_double), t.shape[0]),
                          "mt_case_set_surface")
            ctx.check(lib().mt_case_generate(ctx.h, self.id, C.byref(ms)), "mt_case_generate")
            self._finish(m, schedule, scaling)
            return
        for l in range(self.L + 1):
            for name, sid in SET_IDS.items():
                k = np.ascontiguousarray(m.levels[l].get(name, np.zeros(0, np.uint64)), np.uint64)
                if sid == 6 and not k.size:
                    continue
                ctx.check(lib().mt_case_add_set(ctx.h, self.id, l, sid, _ptr(k, C.c_uint64), k.size), "add_set")
        for b in range(26):
            k = np.ascontiguousarray(m.lat_bc[b], np.uint64)
            ctx.check(lib().mt_case_add_set(ctx.h, self.id, 0, SET_LAT_BC0 + b, _ptr(k, C.c_uint64), k.size),
                      "add_set")
        dk = np.ascontiguousarray(m.dis_keys, np.uint64)
        dr = np.ascontiguousarray(m.dis_rows, np.float64)
        ctx.check(lib().mt_case_set_dis(ctx.h, self.id, _ptr(dk, C.c_uint64), _ptr(dr, C.c_double), dk.size),
                  "set_dis")
        ctx.check(lib().mt_case_build(ctx.h, self.id), "mt_case_build")
        self._finish(m, schedule, scaling)

    def _finish(self, m, schedule, scaling):
        if m.markers is not None:
            self.set_markers(m.markers)
        self.set_schedule(schedule)
        self.set_interface_scaling(scaling)
        self.set_interface_time(self.interface_time)
        for face, u in sorted(getattr(self.case.params, "face_u", {}).items()):
            self.set_face_velocity(face, u)

    def prepare(self):
        """Switch to the fused schedule and build its tables now."""
        self.ctx.check(lib().mt_case_prepare(self.ctx.h, self.id), "mt_case_prepare")
        self.schedule = "fused"

    def transfer(self, dst: Context):
        """Move this case to another context on the same device."""
        nid = C.c_int32()
        self.ctx.check(lib().mt_case_transfer(self.ctx.h, self.id, dst.h, C.byref(nid)), "mt_case_transfer")
        self.ctx = dst
        self.id = nid.value

    def set_markers(self, mk):
        """Upload the Lagrangian markers of a direct-forcing sphere (Markers)."""
        ref = np.ascontiguousarray(mk.ref, np.float64)
        dv = np.ascontiguousarray(mk.dv, np.float64)
        ctr = np.ascontiguousarray(mk.center, np.float64)
        path = np.ascontiguousarray(mk.path, np.float64)
        self.ctx.check(lib().mt_case_set_markers(self.ctx.h, self.id, dv.size, _ptr(ref, C.c_double),
                                                 _ptr(dv, C.c_double), _ptr(ctr, C.c_double), path.shape[0],
                                                 _ptr(path, C.c_double)), "set_markers")

    def set_face_velocity(self, face: int, u):
        """Velocity of boundary face `face` (0..5 = West East South North Bot
        Top); resets that face's boundary cells to feq(rho0, u)."""
        u = np.ascontiguousarray(u, np.float64)
        self.ctx.check(lib().mt_case_set_face_velocity(self.ctx.h, self.id, int(face), _ptr(u, C.c_double)),
                       "set_face_velocity")

    def set_interface_scaling(self, scaling: str):
        """"reference" (the reference's factors) or "standard" (stress-continuous)."""
        self.ctx.check(lib().mt_case_set_interface_scaling(self.ctx.h, self.id, SCALINGS[scaling]), "set_scaling")
        self.scaling = scaling

    def set_interface_time(self, mode: str):
        """"reference" (explosion in the first substep only), "hold" (both
        substeps, from the parent's post-collision state) or "extrap" (the
        second from the parent state extrapolated to the half step)."""
        self.ctx.check(lib().mt_case_set_interface_time(self.ctx.h, self.id, ITIMES[mode]), "set_interface_time")
        self.interface_time = mode

    def set_schedule(self, schedule: str):
        self.ctx.check(lib().mt_case_set_schedule(self.ctx.h, self.id, SCHEDULES[schedule]), "set_schedule")
        self.schedule = schedule

    # ---- D_map_define-style access ------------------------------------
    def size(self, level):
        n = C.c_int64()
        self.ctx.check(lib().mt_case_level_size(self.ctx.h, self.id, level, C.byref(n)), "level_size")
        return n.value

    def keys(self, level):
        n = self.size(level)
        k = np.zeros(n, np.uint64)
        t = np.zeros(n, np.uint32)
        self.ctx.check(lib().mt_case_get_keys(self.ctx.h, self.id, level, _ptr(k, C.c_uint64), _ptr(t, C.c_uint32)),
                       "get_keys")
        return k, t

    def find(self, level, keys):
        keys = np.ascontiguousarray(keys, np.uint64)
        out = np.zeros(keys.size, np.int64)
        self.ctx.check(lib().mt_find(self.ctx.h, self.id, level, _ptr(keys, C.c_uint64), keys.size,
                                     _ptr(out, C.c_int64)), "mt_find")
        return out

    def neighbors(self, level):
        n = self.size(level)
        out = np.zeros((self.q - 1, n), np.int32)
        self.ctx.check(lib().mt_case_get_neighbors(self.ctx.h, self.id, level, _ptr(out, C.c_int32)), "neighbors")
        return out

    # ---- state --------------------------------------------------------
    def initial_equilibrium(self, rho0, u0):
        u = np.ascontiguousarray(u0, np.float64)
        self.ctx.check(lib().mt_case_init_equilibrium(self.ctx.h, self.id, float(rho0), _ptr(u, C.c_double)),
                       "init_equilibrium")

    def set_populations(self, level, f, fcol=None):
        f = np.ascontiguousarray(f, np.float64)
        fc = f if fcol is None else np.ascontiguousarray(fcol, np.float64)
        self.ctx.check(lib().mt_case_set_populations(self.ctx.h, self.id, level, _ptr(f, C.c_double),
                                                     _ptr(fc, C.c_double)), "set_populations")

    def populations(self, level):
        n = self.size(level)
        f = np.zeros((self.q, n))
        fc = np.zeros((self.q, n))
        self.ctx.check(lib().mt_case_get_populations(self.ctx.h, self.id, level, _ptr(f, C.c_double),
                                                     _ptr(fc, C.c_double)), "get_populations")
        return f, fc

    def macros(self, level):
        n = self.size(level)
        rho = np.zeros(n)
        u = np.zeros((3, n))
        self.ctx.check(lib().mt_case_get_macros(self.ctx.h, self.id, level, _ptr(rho, C.c_double),
                                                _ptr(u, C.c_double)), "get_macros")
        return rho, u

    # ---- the reference call surface ------------------------------------
    def calculateMacros(self, level=None):
        levels = range(self.L + 1) if level is None else [level]
        for l in levels:
            self.ctx.check(lib().mt_calculate_macros(self.ctx.h, self.id, l), "calculateMacros")

    def collide(self, level):
        self.ctx.check(lib().mt_collide(self.ctx.h, self.id, level), "collide")

    def stream(self, level):
        self.ctx.check(lib().mt_stream(self.ctx.h, self.id, level), "stream")

    def AMR_transDDF_explosion(self, level):
        self.ctx.check(lib().mt_explosion(self.ctx.h, self.id, level), "explosion")

    def AMR_transDDF_coalescence(self, level):
        self.ctx.check(lib().mt_coalescence(self.ctx.h, self.id, level), "coalescence")

    FACES = {"West": 0, "East": 1, "South": 2, "North": 3, "Bot": 4, "Top": 5}

    def applyBoundaryCondition(self, face=None, position="AfterStream"):
        """All faces in the reference's order, or one face by name."""
        if position != "AfterStream":
            raise MTError("only the AfterStream position exists on the live boundary path")
        if face is None:
            self.ctx.check(lib().mt_apply_bc(self.ctx.h, self.id), "applyBoundaryCondition")
        else:
            self.ctx.check(lib().mt_apply_bc_face(self.ctx.h, self.id, self.FACES[face]), "applyBoundaryCondition")

    def treat(self):
        self.ctx.check(lib().mt_ib_treat(self.ctx.h, self.id), "treat")

    def LBMkernel(self, level=0):
        self.ctx.check(lib().mt_lbm_kernel(self.ctx.h, self.id, level), "LBMkernel")

    def fluidSimulate(self, n_coarse_steps):
        """n coarse steps (graph-replayed); asynchronous on the context stream."""
        self.ctx.check(lib().mt_step(self.ctx.h, self.id, int(n_coarse_steps)), "mt_step")

    def close(self):
        """Release the case's device memory (mt_case_destroy)."""
        if getattr(self, "id", None) is not None and self.ctx.h:
            lib().mt_case_destroy(self.ctx.h, self.id)
        self.id = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def force(self):
        out = np.zeros(4)
        self.ctx.check(lib().mt_get_force(self.ctx.h, self.id, _ptr(out, C.c_double)), "get_force")
        return out

    def tune_bricks(self):
        """Time every form of every brick level's fused pass (0 one cell per
        lane step, 1 a packed pair, 2 one cell with more registers, 3 the
        lane's two cells unrolled together) and keep the fastest per level; returns (form per level, -1
        without bricks; ms per launch [level][form], -1 where not timed)."""
        v = np.zeros(self.L + 1, np.int32)
        ms = np.zeros((self.L + 1, BRICK_FORMS), np.float32)
        self.ctx.check(lib().mt_case_tune_bricks(self.ctx.h, self.id, _ptr(v, C.c_int32), _ptr(ms, C.c_float)),
                       "mt_case_tune_bricks")
        return v, ms

    def set_brick_forms(self, forms):
        """Run each level's brick pass in the given form (a negative entry
        keeps the level's form); FP64 storage has forms 0 and 3."""
        v = np.ascontiguousarray(forms, np.int32)
        if v.shape != (self.L + 1,):
            raise ValueError(f"one form per level: {self.L + 1} entries")
        self.ctx.check(lib().mt_case_set_brick_forms(self.ctx.h, self.id, _ptr(v, C.c_int32)),
                       "mt_case_set_brick_forms")

    def reduce_levels(self):
        """FP64 device sums per level (rows 0..L) and volume-weighted over all
        levels (row L+1): columns mass, x/y/z momentum, kinetic energy."""
        out = np.zeros((self.L + 2, 5))
        self.ctx.check(lib().mt_case_reduce_levels(self.ctx.h, self.id, _ptr(out, C.c_double)), "reduce_levels")
        return out

    def steps(self) -> int:
        """Coarse steps taken (mt_case_get_step)."""
        out = np.zeros(1, np.int64)
        self.ctx.check(lib().mt_case_get_step(self.ctx.h, self.id, _ptr(out, C.c_int64)), "mt_case_get_step")
        return int(out[0])

    def save_checkpoint(self, path):
        """The case's state to `path` (.npz): per level its sorted keys and
        FP64 populations f and fcol, the coarse steps taken and, for a
        direct-forcing case, the force field of its band.  Loading it
        into a case of the same lattice and storage (load_checkpoint) and
        stepping on gives what stepping on here gives, bit for bit in FP64
        (the reference and hold interface times; the extrapolated one keeps
        parent values of the previous step that are not saved)."""
        arrays = {"meta": np.array([self.q, self.L, _storage_code(self.storage or self.case.params.storage), self.steps()], np.int64)}
        for l in range(self.L + 1):
            keys, _ = self.keys(l)
            f, fcol = self.populations(l)
            arrays[f"keys{l}"], arrays[f"f{l}"], arrays[f"fcol{l}"] = keys, f, fcol
        if self.case.params.ib_method == "DF":
            # the force the band's next collision takes
            acc = np.zeros((3, self.size(self.L)), np.int64)
            self.ctx.check(lib().mt_case_get_df_force_field(self.ctx.h, self.id, _ptr(acc, C.c_int64)),
                           "mt_case_get_df_force_field")
            arrays["df_force"] = acc
        np.savez(path, **arrays)

    def load_checkpoint(self, path):
        """Restore a state saved by save_checkpoint (same lattice and storage)."""
        z = np.load(path)
        q, L, st, steps = (int(v) for v in z["meta"])
        if (q, L, st) != (self.q, self.L, _storage_code(self.storage or self.case.params.storage)):
            raise ValueError("checkpoint of another model, level count or storage")
        for l in range(L + 1):
            if not np.array_equal(self.keys(l)[0], z[f"keys{l}"]):
                raise ValueError(f"checkpoint of another lattice (level {l})")
        for l in range(L + 1):
            self.set_populations(l, z[f"f{l}"], z[f"fcol{l}"])
        if "df_force" in z.files:
            acc = np.ascontiguousarray(z["df_force"], np.int64)
            self.ctx.check(lib().mt_case_set_df_force_field(self.ctx.h, self.id, _ptr(acc, C.c_int64)),
                           "mt_case_set_df_force_field")
        self.ctx.check(lib().mt_case_set_step(self.ctx.h, self.id, steps), "mt_case_set_step")

    def info(self):
        """infoPrint's diagnostics per level (mt_case_info): rows 0..L,
        columns max |u| and cells with |u| > 1 (lat_f and overlap_F2C), sum
        |u - u_prev|^2 and sum |u|^2 (lat_f; u_prev = the previous call's)."""
        out = np.zeros((self.L + 1, 4))
        self.ctx.check(lib().mt_case_info(self.ctx.h, self.id, _ptr(out, C.c_double)), "mt_case_info")
        return out

    def infoPrint(self, iter_no, file=None):
        """The line LBM_Manager::infoPrint prints (LBM_Manager.cpp:914-979):
        the velocity change since the previous call relative to the velocity,
        per level max |u| / cells above 1, and for a sphere the drag
        coefficient of the mean force per treat() call since the previous
        call (the accumulated force is then reset, as the reference resets its
        sums) with its running average.  Returns the line."""
        import sys
        d = self.info()
        err = float(np.sqrt(d[:, 2].sum()) / np.sqrt(d[:, 3].sum() + 1e-16))
        line = f"[Iter] {iter_no} Velocity error = {err:.6g} | max|v|/nbig:"
        line += "".join(f" L{l}={d[l, 0]:.6g}/{int(d[l, 1])}" for l in range(self.L + 1))
        sphere = getattr(self.case.mesh.spec, "sphere", None)
        f = self.force()
        if sphere is not None and f[3] > 0:
            dia = 2.0 * sphere.radius * (1 << self.L)
            cd = drag_coefficient(f, self.case.params.u_ref, dia)
            self._cd = getattr(self, "_cd", []) + [cd]
            line += (f"  Cd = {cd:.6g}  (Cd_avg = {np.mean(self._cd):.6g}, Fx_lb = {f[0] / f[3]:.6g}, "
                     f"n = {int(f[3])})")
            self.reset_force()
        print(line, file=file or sys.stdout)
        return line

    def remap_from(self, src: "LBM_Manager", counts: bool = True):
        """Carry src's state onto this case's lattice (mt_case_remap); returns
        the cells per level that were copied, taken from an ancestor, taken
        from descendants, or set to equilibrium ((L+1, 4) array), or None
        when counts is False (no read-back)."""
        if not counts:
            self.ctx.check(lib().mt_case_remap(self.ctx.h, self.id, src.id, None), "mt_case_remap")
            return None
        out = np.zeros(4 * (self.L + 1), np.int64)
        self.ctx.check(lib().mt_case_remap(self.ctx.h, self.id, src.id, _ptr(out, C.c_int64)), "mt_case_remap")
        return out.reshape(self.L + 1, 4)

    def remeshed(self, case: Case, storage: str = None, schedule: str = None) -> "LBM_Manager":
        """A new case on `case`'s lattice (other refinement boxes, a moved
        body's band or markers) carrying this case's state; this case is left
        as it is (close it when done)."""
        new = LBM_Manager(self.ctx, case, storage or self.storage, schedule=schedule or self.schedule,
                          scaling=self.scaling, storage_shift=self.storage_shift)
        new.remap_from(self, counts=False)
        return new

    def force_async(self):
        """Enqueue a copy of the accumulated force (read it with force_copied
        once a marker recorded after this call is done)."""
        self.ctx.check(lib().mt_case_force_async(self.ctx.h, self.id), "mt_case_force_async")

    def force_copied(self):
        out = np.zeros(4)
        self.ctx.check(lib().mt_case_force_copied(self.ctx.h, self.id, _ptr(out, C.c_double)), "mt_case_force_copied")
        return out

    def finite_copied(self) -> bool:
        """Whether the state was finite when force_async was enqueued (its
        guard flags arrive with the force copy)."""
        rc = lib().mt_case_status_copied(self.ctx.h, self.id)
        if rc == -5:
            return False
        self.ctx.check(rc, "mt_case_status_copied")
        return True

    def reset_force(self):
        self.ctx.check(lib().mt_reset_force(self.ctx.h, self.id), "reset_force")

    def status(self):
        """Raise MTError (MT_ERR_NONFINITE / MT_ERR_MESH) if the device
        guard finds a problem; returns None when healthy."""
        self.ctx.check(lib().mt_case_status(self.ctx.h, self.id), "mt_case_status")


class Batch:
    """Independent multi-level cases stepped together (mt_batch_*): one
    batched brick pass per level, substep and model family; each member ends
    a step exactly where it would stepped alone under the fused schedule."""

    def __init__(self, ctx: Context, managers=()):
        self.ctx = ctx
        bid = C.c_int32()
        ctx.check(lib().mt_batch_create(ctx.h, C.byref(bid)), "mt_batch_create")
        self.id = bid.value
        self.members = []
        for m in managers:
            self.add(m)

    def add(self, mgr):
        self.ctx.check(lib().mt_batch_add(self.ctx.h, self.id, mgr.id), "mt_batch_add")
        mgr.schedule = "fused"
        self.members.append(mgr)

    def remove(self, mgr):
        self.ctx.check(lib().mt_batch_remove(self.ctx.h, self.id, mgr.id), "mt_batch_remove")
        self.members.remove(mgr)

    def __len__(self):
        n = C.c_int32()
        self.ctx.check(lib().mt_batch_size(self.ctx.h, self.id, C.byref(n)), "mt_batch_size")
        return n.value

    def step(self, n=1):
        self.ctx.check(lib().mt_batch_step(self.ctx.h, self.id, int(n)), "mt_batch_step")

    def close(self):
        if getattr(self, "id", None) is not None and self.ctx.h:
            lib().mt_batch_destroy(self.ctx.h, self.id)
        self.id = None


class DenseCase:
    """Dense periodic Morton cube (uniform single level), any storage."""

    def __init__(self, ctx: Context, case: Case, storage: str = None):
        self.ctx = ctx
        self.case = case
        self.q = case.params.q
        d = make_desc(case, storage)
        cid = C.c_int32()
        ctx.check(lib().mt_case_create_dense(ctx.h, C.byref(d), C.byref(cid)), "mt_case_create_dense")
        self.id = cid.value
        n = C.c_int64()
        ctx.check(lib().mt_case_level_size(ctx.h, self.id, 0, C.byref(n)), "level_size")
        self.n = n.value

    def init_fields(self, rho, ux, uy, uz):
        arrs = [np.ascontiguousarray(a, np.float64).ravel() for a in (rho, ux, uy, uz)]
        self.ctx.check(lib().mt_case_init_fields(self.ctx.h, self.id, *[_ptr(a, C.c_double) for a in arrs]),
                       "init_fields")
        return arrs

    def init_fields_ptr(self, rho_ptr, ux_ptr, uy_ptr, uz_ptr):
        """Same as init_fields from raw host pointers (pinned buffers)."""
        cast = lambda p: C.cast(C.c_void_p(p), C.POINTER(C.c_double))  # noqa: E731
        self.ctx.check(lib().mt_case_init_fields(self.ctx.h, self.id, cast(rho_ptr), cast(ux_ptr), cast(uy_ptr),
                                                 cast(uz_ptr)), "init_fields")

    def set_populations(self, f):
        f = np.ascontiguousarray(f, np.float64)
        self.ctx.check(lib().mt_case_set_populations(self.ctx.h, self.id, 0, _ptr(f, C.c_double), None),
                       "set_populations")

    def populations(self):
        f = np.zeros((self.q, self.n))
        fc = np.zeros((self.q, self.n))
        self.ctx.check(lib().mt_case_get_populations(self.ctx.h, self.id, 0, _ptr(f, C.c_double),
                                                     _ptr(fc, C.c_double)), "get_populations")
        return f, fc

    def macros(self):
        rho = np.zeros(self.n)
        u = np.zeros((3, self.n))
        self.ctx.check(lib().mt_case_get_macros(self.ctx.h, self.id, 0, _ptr(rho, C.c_double), _ptr(u, C.c_double)),
                       "get_macros")
        return rho, u

    def macros_ptr(self, rho_ptr, u_ptr):
        cast = lambda p: C.cast(C.c_void_p(p), C.POINTER(C.c_double))  # noqa: E731
        self.ctx.check(lib().mt_case_get_macros(self.ctx.h, self.id, 0, cast(rho_ptr), cast(u_ptr)), "get_macros")

    def reduce(self):
        out = np.zeros(5)
        self.ctx.check(lib().mt_case_reduce(self.ctx.h, self.id, _ptr(out, C.c_double)), "reduce")
        return dict(mass=out[0], momentum=out[1:4].copy(), kinetic_energy=out[4])

    def step(self, n=1):
        self.ctx.check(lib().mt_step(self.ctx.h, self.id, int(n)), "mt_step")

    def tune(self):
        """Pick the fused kernel's block size (state unchanged); returns
        (block, {block: ms per launch})."""
        best = C.c_int32()
        ms = (C.c_float * 4)(*([-1.0] * 4))
        self.ctx.check(lib().mt_case_tune(self.ctx.h, self.id, C.byref(best), ms), "mt_case_tune")
        # candidates the kernel is not built for (paired 16-bit LBGK: at most 256 threads) are left out
        return best.value, {b: round(float(v), 5) for b, v in zip((128, 256, 512, 1024), ms) if v >= 0.0}

    def close(self):
        if getattr(self, "id", None) is not None and self.ctx.h:
            lib().mt_case_destroy(self.ctx.h, self.id)
        self.id = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def drag_coefficient(force4, u_lattice, diameter_finest_cells, rho=1.0):
    """Cd = 2 F / (rho U^2 pi d^2 / 4) with F the mean momentum-exchange
    force per treat() call (force4 = fx, fy, fz, number of calls, as
    mt_get_force returns it), U the boundary velocity in level-0 lattice
    units and d the sphere diameter in finest cells -- the formula of
    LBM_Manager::infoPrint (LBM_Manager.cpp:964-979)."""
    fx = force4[0] / max(force4[3], 1.0)
    area = np.pi * diameter_finest_cells * diameter_finest_cells / 4.0
    return 2.0 * fx / (rho * u_lattice * u_lattice * area)


def morton_order_fields(n_edge, *fields):
    """Reorder (x, y, z)-indexed cube fields into Morton (sorted key) order."""
    from .lattice import morton_encode
    idx = np.arange(n_edge)
    X, Y, Z = np.meshgrid(idx, idx, idx, indexing="ij")
    order = np.argsort(morton_encode(X.ravel(), Y.ravel(), Z.ravel()), kind="stable")
    return [np.ascontiguousarray(f.ravel()[order]) for f in fields]
