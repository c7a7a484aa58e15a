/*
 * mt_lbm.h -- C ABI of libmtlbm, the B200 (sm_100a) implementation of the
 * multi-level lattice-Boltzmann time step of MortonTrieCode-CAD2025/
 * mortonTrie_AMR.
 *
 * Every function returns an int status (MT_OK or a negative MT_ERR_* code);
 * none aborts the process.  mt_last_error() gives a readable message for the
 * last failure on a context.  Device memory is owned by the context; host
 * buffers are owned by the caller.  Populations cross the boundary as FP64
 * structure-of-arrays [Q][n], n cells of one level in ascending Morton-key
 * order (the order mt_case_get_keys returns).
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   D_map_define<T>            header/Grid_Class.h:116-137, header/user.h:18-45
 *   Lat_Manager index sets     header/Lat_Manager.hpp:245-316
 *   LBM_Manager                header/LBM_Manager.hpp:25-119
 *   Collision_Model::collide   header/lbm_kernel/Collision_Manager.hpp:73-97
 *   Stream_Model::stream       header/lbm_kernel/Stream_Manager.hpp:12-37
 *   ComplexBoundary_Model      header/ComplexBoundary_Manager.hpp:16-46
 *   D3Q19_BC_Strategy/Manager  header/BC/D3Q19_BC_Manager.hpp:15-263
 */
#ifndef MT_LBM_H
#define MT_LBM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MT_MAX_LEVELS 8

/* status codes */
#define MT_OK 0
#define MT_ERR_ARG (-1)      /* bad argument or unsupported combination */
#define MT_ERR_CUDA (-2)     /* a CUDA call failed */
#define MT_ERR_STATE (-3)    /* call out of order (e.g. step before build) */
#define MT_ERR_MESH (-4)     /* index sets violate the contract (missing child / neighbour) */
#define MT_ERR_NONFINITE (-5) /* the device guard found a NaN/Inf population */

/* lattice index sets, Lat_Manager.hpp:245-316 */
#define MT_SET_LAT_F 0
#define MT_SET_OVERLAP_F2C 1
#define MT_SET_OVERLAP_C2F 2
#define MT_SET_GHOST_C2F 3
#define MT_SET_GHOST_F2C 4
#define MT_SET_LAT_SF 5
#define MT_SET_IB_BAND 6  /* finest-level cells the markers' forcing can reach (MT_IB_DF; no reference counterpart) */
#define MT_SET_LAT_BC0 16 /* MT_SET_LAT_BC0 + b, b = 0..25 in Bdry_Type order (D3Q19_BC_Manager.hpp:25-53) */

#define MT_COLL_LBGK 0     /* Collision_LBGK, lbm_kernel/Collision_Manager.cpp:13-53 */
#define MT_COLL_CUMULANT 1 /* Collision_Cumulant, lbm_kernel/Collision_Cumulant.cpp:22-652 (Q = 27) */
#define MT_IB_DW 0         /* SinglePointInterpolation, distance weighted */
#define MT_IB_FH 1         /* SinglePointInterpolation, Filippova-Haenel */
#define MT_IB_DF 2         /* direct forcing on Lagrangian markers (no reference counterpart) */
#define MT_BC_NEQ 0        /* nonEquilibrumExtrapolation_* (BC/NonEquilibrumExtrapolation.cpp) */
#define MT_BC_ZOUHE_OUTFLOW 1 /* velocity inlet on West, zero-gradient outflow on East */
/* Zou-He velocity inlet with Hecht-Harting corrections on West (formula family of
   BC/ZouHe_Velocity.cpp:81-93,170-199), five-population outflow on East
   (BC/Outflow.cpp:39-52); wet nodes on the boundary shell, D3Q19 LBGK, phase schedule */
#define MT_BC_ZOUHE_HH 2
#define MT_PULL_REFERENCE 0   /* f_q(x) = fcol_q(x + e_q), Stream_Manager.cpp:43-76 */
#define MT_PULL_TEXTBOOK 1    /* f_q(x) = fcol_q(x - e_q) */
#define MT_STORE_F64 0
#define MT_STORE_F32 1  /* FP32 storage of f - s_q (u_shift below), FP32 arithmetic */
#define MT_STORE_F16 2  /* FP16 storage of f - s_q, FP32 arithmetic */
#define MT_STORE_BF16 3 /* BF16 storage of f - s_q, FP32 arithmetic */
#define MT_SCHED_PHASES 0 /* the reference's phase order: collide, stream, ... as separate passes */
#define MT_SCHED_FUSED 1  /* stream of one substep fused with the collision of the next (same results) */
#define MT_SCHED_FUSED_LISTS 2 /* MT_SCHED_FUSED over cell lists and the neighbour table, no 4x4x4 bricks */
#define MT_SCALE_REFERENCE 0 /* explosion x 2 tau_f / tau_c, coalescence x tau_c / (2 tau_f): LBM_Manager.cpp:1065, 1137 */
#define MT_SCALE_STANDARD 1  /* stress-continuous rescaling: fneq_f = tau_f / (2 tau_c) fneq_c and its inverse */
#define MT_ITIME_REFERENCE 0 /* fine level explodes in its first substep only: LBM_Simulator.cpp:47-51 */
#define MT_ITIME_HOLD 1      /* in both substeps, from the parent's post-collision state of the coarse step */
#define MT_ITIME_EXTRAP 2    /* second substep from that state extrapolated to the half step */

/* Case description: the switches the reference hard-codes in
 * LBM_Manager::LBM_Manager (LBM_Manager.cpp:32-95) and its per-level
 * relaxation times from LBM_Manager::setUnit (LBM_Manager.cpp:763-844). */
typedef struct mt_case_desc {
    int32_t q;                 /* 19 or 27 */
    int32_t max_level;         /* C_max_level, 0 .. MT_MAX_LEVELS-1 */
    int32_t collision;         /* MT_COLL_* */
    int32_t ib_method;         /* MT_IB_* */
    int32_t bc_mode;           /* MT_BC_* */
    int32_t stream_convention; /* MT_PULL_* */
    int32_t storage;           /* MT_STORE_*; FP64 is the reference precision (bit-exact) */
    int32_t periodic[3];       /* per axis: 1 wraps neighbours (no reference counterpart; BC/Periodic.cpp is dead code) */
    int64_t extent0[3];        /* level-0 cells per axis */
    double tau[MT_MAX_LEVELS]; /* LBM_Manager::tau */
    double rho0;               /* U_rho0 / CF_Rho */
    double u_bc[3];            /* boundary velocity in lattice units (input_v / CF_U) */
    /* Storage shift velocity u_s of the reduced storages, per level (no
     * reference counterpart): FP32/FP16/BF16 keep f_k - feq_k(1, u_s) instead
     * of f_k, so the stored deviations stay small where the flow is near u_s
     * (the inlet velocity on the far-field levels of a channel flow; the
     * level holding a wall is better kept at zero, since the wall
     * populations are near w).  All zero: f_k - w_k.  FP64 stores f. */
    double u_shift[MT_MAX_LEVELS][3];
} mt_case_desc;

typedef struct mt_ctx mt_ctx;

/* ---- context ---------------------------------------------------------- */
/* A context on `device` with a stream of its own.  It also sets the release
 * threshold of the device's default memory pool (cudaDeviceGetDefaultMemPool)
 * to unlimited, so memory freed by stream-ordered frees stays in the pool for
 * the next case build instead of being returned at every synchronisation;
 * that pool is shared by every user of cudaMallocAsync in the process. */
int mt_create(int32_t device, mt_ctx **out);
int mt_destroy(mt_ctx *ctx);
const char *mt_last_error(const mt_ctx *ctx);
/* run all work of this context on a caller-owned cudaStream_t (NULL: own stream) */
int mt_set_stream(mt_ctx *ctx, void *cuda_stream);
int mt_synchronize(mt_ctx *ctx);
/* Give the context's own stream the device's highest (high != 0) or lowest
 * scheduling priority (no reference counterpart): a context that builds
 * cases while another runs long batches gets its short kernels scheduled
 * first.  Synchronises the context; MT_ERR_STATE on a caller's stream. */
int mt_set_priority(mt_ctx *ctx, int32_t high);
/* kernels launched by this context so far (graph replays count their nodes) */
int mt_launch_count(const mt_ctx *ctx, int64_t *out);

/* ---- case setup: LBM_Manager::LBM_Manager + allocMacrosAndDDF --------- */
int mt_case_create(mt_ctx *ctx, const mt_case_desc *desc, int32_t *case_id);
/* Dense periodic Morton cube (no counterpart in the reference): max_level 0,
 * all axes periodic, equal power-of-two extents; every cell is lat_f and the
 * key set is generated on the device. */
int mt_case_create_dense(mt_ctx *ctx, const mt_case_desc *desc, int32_t *case_id);
int mt_case_destroy(mt_ctx *ctx, int32_t case_id);
/* add keys to one index set of one level (Lat_Manager::lat_f[l].insert ...) */
int mt_case_add_set(mt_ctx *ctx, int32_t case_id, int32_t level, int32_t set_id, const uint64_t *keys, int64_t n);
/* Lat_Manager::dis: finest-level keys (ascending) and Q-1 wall distances each */
int mt_case_set_dis(mt_ctx *ctx, int32_t case_id, const uint64_t *keys, const double *rows, int64_t n);
/* Box-and-sphere lattice classified on the device (no reference counterpart:
 * the reference voxelises an STL in Lat_Manager::voxelize, Lat_Voxelize.cpp
 * :17-733).  Produces the index-set contract of Lat_Manager.hpp:245-316 for
 * nested refinement boxes: the level-0 boundary shell split into the 26
 * lat_bc sets (Lat_Voxelize.cpp:242-288), F2C = the 1-cell shell of each
 * refinement box, C2F = the 2-cell shell of each refined level, the ghost
 * layers from the Q neighbours (Lat_Voxelize.cpp:676-733), and for a sphere
 * either the voxelised solid with its wall distances (Lat_Voxelize.cpp
 * :1252-1285) or the direct-forcing band. */
typedef struct mt_mesh_spec {
    int64_t coarse[3];                   /* level-0 cells per axis (the case's extent0) */
    int32_t boundary_bc[3];              /* 1: boundary shell on this axis, 0: periodic (the case's periodic[] inverted) */
    int32_t has_refine[MT_MAX_LEVELS];   /* level l < max_level is refined: 1 in the box refine_lo/hi[l],
                                            2 in the region of level l + 1 set by mt_case_set_region (an
                                            octree: every refined level then takes a region) */
    int64_t refine_lo[MT_MAX_LEVELS][3]; /* the box [lo, hi) in level-l cells */
    int64_t refine_hi[MT_MAX_LEVELS][3];
    int32_t sphere;                      /* 0 none, 1 solid + wall distances, 2 forcing band (MT_IB_DF),
                                            3 the triangulated surface of mt_case_set_surface (solid + wall distances) */
    int32_t pad;
    double center[3];                    /* coarse-cell units from the box corner */
    double radius;                       /* coarse cells */
    double osc_amplitude;                /* band of a sphere oscillating along y: amplitude in coarse cells */
    double band_slack;                   /* extra inner band depth in coarse cells */
} mt_mesh_spec;

/* Closed triangulated solid surface for mt_case_generate with sphere = 3
 * (an STL body, Shape::geofile_stl, Shape.cpp:341-470): tri[n][3][3] vertex
 * coordinates in coarse-cell units.  A finest-level cell is solid when its
 * centre lies inside (odd number of crossings of the +x line from the centre,
 * edges shared by two triangles counted once); the wall distance of each
 * link of a fluid cell is its nearest crossing with a triangle
 * (Shape::intersect_line_with_triangle, Shape.cpp:809-843, edges included)
 * normalised by the link length and kept in [0, 1]
 * (Lat_Manager::compute_distance, Lat_Voxelize.cpp:1252-1285). */
int mt_case_set_surface(mt_ctx *ctx, int32_t case_id, const double *tri, int64_t n);
/* Refinement region of `level` (1..max_level) for mt_case_generate with
 * has_refine[level - 1] = 2 (refinement made from the body instead of boxes,
 * the octree of Grid_Manager::generate_inner, Grid_Manager.cpp:136-454, with
 * the intermediate levels its generate_intermediate leaves empty,
 * :99-102): the level-(level - 1) cells refined to `level`, a dense mask
 * mask[(i * shape[1] + j) * shape[2] + k] != 0 for cell lo + (i, j, k).  The
 * level's cells are the children of the region; its overlap_C2F cells are
 * the children of the region's cells with one of their 26 neighbours outside
 * it, which are the coarser level's overlap_F2C cells; the rest of the
 * region is stored on the finer level only.  The box [lo, lo + shape) must
 * lie inside level (level - 1)'s extent; regions must nest 2:1 (each inside
 * the coarser one with room for the interface layers), which
 * mt_case_generate checks as it does for boxes. */
int mt_case_set_region(mt_ctx *ctx, int32_t case_id, int32_t level, const int64_t *lo, const int64_t *shape,
                       const uint8_t *mask);
/* generate the case's sets from spec and build it (replaces mt_case_add_set,
 * mt_case_set_dis and mt_case_build); MT_ERR_MESH with the host mesher's
 * messages when the boxes or the sphere break the contract */
int mt_case_generate(mt_ctx *ctx, int32_t case_id, const mt_mesh_spec *spec);
/* Carry the state of case src onto case dst, a lattice of the same model
 * (Q, levels, level-0 extent, storage) built from other refinement boxes: moving the
 * refinement with a body (the reference's dynamic remeshing,
 * Grid_Manager_dynamic.cpp, is not compiled in; no counterpart in its step).
 * Each cell of dst takes f and fcol from src: the same key on the same level
 * as they are (bit for bit); else from its ancestor on the nearest coarser
 * level holding one, the non-equilibrium part rescaled as an explosion; else
 * from the mean of its descendants on the nearest finer level holding any,
 * rescaled as a coalescence; else the equilibrium
 * (rho0, u_bc).  Solid cells of dst hold zeros; a fluid cell of dst that is
 * solid in src takes the equilibrium at rest.  The interface factors are
 * dst's.  dst's direct-forcing step
 * counter follows src's (markers are dst's own).  counts (nullable) receives
 * [4 * level + kind] cells of each kind 0..3 in that order.  Neither case may
 * be in a batch. */
int mt_case_remap(mt_ctx *ctx, int32_t dst_case, int32_t src_case, int64_t *counts);
/* device build: radix sort + unique of the keys, set tags, neighbour table
 * by binary search of the Morton neighbour keys (Morton_Assist::find_neighbor
 * + D_map_define::find), explosion/coalescence child tables, IB list */
int mt_case_build(mt_ctx *ctx, int32_t case_id);
int mt_case_level_size(mt_ctx *ctx, int32_t case_id, int32_t level, int64_t *n);
int mt_case_get_keys(mt_ctx *ctx, int32_t case_id, int32_t level, uint64_t *keys, uint32_t *tags);
/* neighbour table [(Q-1)][n]: index of the cell at key + e_k, or -1 */
int mt_case_get_neighbors(mt_ctx *ctx, int32_t case_id, int32_t level, int32_t *nbr);
/* D_map_define::find in bulk: index of each key on the level, or -1 */
int mt_find(mt_ctx *ctx, int32_t case_id, int32_t level, const uint64_t *keys, int64_t n, int64_t *idx);

/* ---- state ------------------------------------------------------------ */
/* reference initial state (LBM_Manager.cpp:482-592, 296-304): f = fcol =
 * feq(rho0, u0) on every stored cell, zero on solid cells */
int mt_case_init_equilibrium(mt_ctx *ctx, int32_t case_id, double rho0, const double *u0);
/* f = fcol = feq(rho_i, u_i) per cell from host fields [n] (dense path) */
int mt_case_init_fields(mt_ctx *ctx, int32_t case_id, const double *rho, const double *ux, const double *uy,
                        const double *uz);
int mt_case_set_populations(mt_ctx *ctx, int32_t case_id, int32_t level, const double *f, const double *fcol);
int mt_case_get_populations(mt_ctx *ctx, int32_t case_id, int32_t level, double *f, double *fcol);
/* density [n] and velocity [3][n] of a level (density/velocity maps of User) */
int mt_case_get_macros(mt_ctx *ctx, int32_t case_id, int32_t level, double *rho, double *u);
/* FP64 reductions over the stepped cells: out[5] = mass, x/y/z momentum,
   kinetic energy sum of |j|^2 / (2 rho).  Dense path: every cell.  Multi-level
   cases: the volume-weighted total of mt_case_reduce_levels (last row). */
int mt_case_reduce(mt_ctx *ctx, int32_t case_id, double *out5);
/* Per-level FP64 reductions of a multi-level case, the device counterpart of
   the per-level scans of LBM_Manager::infoPrint (LBM_Manager.cpp:914-981):
   out[(max_level + 2) * 5]; row l (l = 0 .. max_level) sums mass sum_q f_q,
   momentum sum_q f_q e_q and |j|^2 / (2 rho) over level l's lat_f and
   overlap_F2C cells (the cells calculateMacros visits), from the streamed f
   widened to FP64 (storage shift added in FP64); row max_level + 1 is
   sum_l 8^-l row_l (a level-l cell is 8^-l coarse cells; the F2C cells stand
   for the region their C2F children cover).  Dense cases: two equal rows.
   Each row is summed in a fixed order (run to run identical). */
int mt_case_reduce_levels(mt_ctx *ctx, int32_t case_id, double *out);
/* The diagnostics LBM_Manager::infoPrint prints each coarse step
   (LBM_Manager.cpp:914-979), from the end-of-step macros on the device:
   out[4 * (max_level + 1)], per level l: out[4l] the largest |u| and
   out[4l + 1] the number of cells with |u| > 1 over lat_f and overlap_F2C
   (a NaN velocity counts in neither, as in the reference's comparisons);
   over lat_f, out[4l + 2] = sum |u - u_prev|^2 and out[4l + 3] = sum |u|^2,
   the reference's velocity error being sqrt(sum_l out[4l + 2] /
   sum_l out[4l + 3]).  u_prev is the velocity the previous mt_case_info call
   of the case saw (the reference keeps the one of the level's last
   substep); the first call reports 0.  The drag part of the line is
   mt_get_force.  Multi-level cases; synchronises the stream. */
int mt_case_info(mt_ctx *ctx, int32_t case_id, double *out);
/* Allocation-free variant of mt_case_reduce; no reference counterpart (the
   reference has no device-side reduction).  For callers that must not allocate
   device memory during the call (a host that budgets the GPU's memory up front
   for its cases).  Same outputs and kernels; the scratch is a static device
   array of 640 KiB, so cases above 4,194,304 cells return MT_ERR_ARG.  Calls
   that overlap in time on one device race on that array: serialise them.  The
   first call on a device does a one-time set-up (looks up the array's address
   with that device current, then makes the caller's current device current
   again); make it before any stream capture.  Synchronises the stream. */
int mt_case_reduce_noalloc(mt_ctx *ctx, int32_t case_id, double *out5);

/* ---- the reference call surface --------------------------------------- */
int mt_calculate_macros(mt_ctx *ctx, int32_t case_id, int32_t level); /* LBM_Manager::calculateMacros(level) */
int mt_collide(mt_ctx *ctx, int32_t case_id, int32_t level);          /* Collision_Model::collide(level) */
int mt_stream(mt_ctx *ctx, int32_t case_id, int32_t level);           /* ABPatternPull::stream(level) */
int mt_explosion(mt_ctx *ctx, int32_t case_id, int32_t level);        /* LBM_Manager::AMR_transDDF_explosion */
int mt_coalescence(mt_ctx *ctx, int32_t case_id, int32_t level);      /* LBM_Manager::AMR_transDDF_coalescence */
int mt_apply_bc(mt_ctx *ctx, int32_t case_id);                        /* applyBoundaryCondition(face, "AfterStream") x 6 */
/* one face group: 0 West, 1 East, 2 South, 3 North, 4 Bot, 5 Top
 * (D3Q19_BoundaryCondtion_Manager::applyBoundaryCondition, D3Q19_BC_Manager.hpp:220-244) */
int mt_apply_bc_face(mt_ctx *ctx, int32_t case_id, int32_t face);
int mt_ib_treat(mt_ctx *ctx, int32_t case_id);                        /* ComplexBoundary_Model::treat */
int mt_lbm_kernel(mt_ctx *ctx, int32_t case_id, int32_t level);       /* LBM_Manager::LBMkernel(level) */
/* n coarse steps of LBM_Manager::fluidSimulate (LBM_Simulator.cpp:11-17):
 * LBMkernel(0) then calculateMacros() on every level, replayed from a CUDA
 * graph; asynchronous on the context stream */
int mt_step(mt_ctx *ctx, int32_t case_id, int32_t n_coarse_steps);
/* Coarse steps the case has taken through mt_step / mt_batch_step (no
 * reference counterpart; with mt_case_get/set_populations the state of a
 * checkpoint).  mt_case_set_step restores the count, and for a
 * direct-forcing case the markers' position on their path, which follows
 * the finest substeps taken; the other cases' steps do not depend on it. */
int mt_case_get_step(mt_ctx *ctx, int32_t case_id, int64_t *coarse_steps);
int mt_case_set_step(mt_ctx *ctx, int32_t case_id, int64_t coarse_steps);
/* The direct-forcing body-force density of the finest level's cells
 * (MT_IB_DF; fixed point, units of 2^-32), [3][n] in the level's key order
 * (no reference counterpart).  Between coarse steps it holds the force the
 * forcing band's next collision takes, so a checkpoint of a direct-forcing
 * case saves and restores it beside the populations and the step count.
 * MT_ERR_STATE for other cases. */
int mt_case_get_df_force_field(mt_ctx *ctx, int32_t case_id, int64_t *out);
int mt_case_set_df_force_field(mt_ctx *ctx, int32_t case_id, const int64_t *in);
/* Health check after a run of steps: scans every population for NaN/Inf
 * (the reference prints NaN diagnostics each substep, LBM_Simulator.cpp:33-86)
 * and reports errors the step kernels raised.  MT_OK, MT_ERR_NONFINITE or
 * MT_ERR_MESH; synchronises the context stream. */
int mt_case_status(mt_ctx *ctx, int32_t case_id);
/* Autotuner of the dense path (no reference counterpart): times the fused
 * kernel at 128, 256, 512 and 1024 threads per block on the case's own state
 * (writing only the scratch array, so the state is unchanged) and keeps the
 * fastest; ms_per_candidate (nullable) receives the mean launch time of each
 * candidate the kernel is built for (the paired 16-bit LBGK kernel: 128 and
 * 256 only; the other slots are left unwritten). */
int mt_case_tune(mt_ctx *ctx, int32_t case_id, int32_t *best_block, float *ms_per_candidate);
/* Forms of the multi-level fused brick pass (no reference counterpart):
 * 0: one cell per lane step at 8 resident 128-thread blocks per SM (FP32: 7),
 *    the default;
 * 3: the lane's two cells in one unrolled sequence, so that the second
 *    cell's gathers overlap the first cell's collision, at 6 blocks;
 * for FP32 / FP16 / BF16 storage also
 * 1: the two cells together in packed FP32 pair arithmetic at 4 blocks,
 * 2: form 0 at 6 blocks with more registers per thread.
 * Forms 0, 2 and 3 compute the same values bit for bit. */
#define MT_BRICK_FORMS 4
/* Project autotuner of the multi-level fused brick pass: times each brick
 * level's pass in each of its forms on the case's own bricks, without
 * changing the state, and keeps the fastest per level for the fused steps
 * that follow.  variant[max_level + 1]: the form kept (-1 for a level without
 * bricks); ms[MT_BRICK_FORMS * (max_level + 1)]: ms per launch of each form
 * (-1 if not timed).  Either may be NULL.  Synchronises the stream; the case
 * keeps its schedule. */
int mt_case_tune_bricks(mt_ctx *ctx, int32_t case_id, int32_t *variant, float *ms);
/* Sets the brick pass form of each level (form[max_level + 1]; a negative
 * entry keeps the level's form), e.g. one a previous mt_case_tune_bricks
 * picked.  MT_ERR_ARG for a form outside 0..MT_BRICK_FORMS-1 or one the
 * storage does not have (FP64: 0 and 3). */
int mt_case_set_brick_forms(mt_ctx *ctx, int32_t case_id, const int32_t *form);
/* Schedule of mt_step for a multi-level case (no reference counterpart):
 * MT_SCHED_PHASES (default) issues the reference's phases one pass each;
 * MT_SCHED_FUSED keeps a second post-collision buffer per level and streams
 * each substep in the same pass as the next substep's macros + collision
 * (LBM_Simulator.cpp:20-229 reordered: the state after every coarse step is
 * the same).  Its fused pass walks 4x4x4 Morton bricks with neighbours
 * computed in shared memory where a level allows it (periodic axes a multiple
 * of 4 cells); MT_SCHED_FUSED_LISTS uses cell lists and the neighbour table
 * everywhere.  The per-phase calls always act on the current buffers. */
int mt_case_set_schedule(mt_ctx *ctx, int32_t case_id, int32_t schedule);
/* Interface rescaling of a multi-level case (no reference counterpart; the
 * reference hard-codes MT_SCALE_REFERENCE, the default).  MT_SCALE_STANDARD
 * is the rescaling that keeps the viscous stress continuous across a 2:1
 * level interface; with the reference's factors the non-equilibrium part is
 * amplified 4x from coarse to fine and flows near tau = 0.5 go unstable. */
int mt_case_set_interface_scaling(mt_ctx *ctx, int32_t case_id, int32_t scaling);
/* When a fine level takes its interface cells from its parent (no reference
 * counterpart; the reference explodes in the first substep only,
 * LBM_Simulator.cpp:47-51,122-125, MT_ITIME_REFERENCE, the default).
 * MT_ITIME_HOLD explodes in the second substep as well, from the same parent
 * values (the parent has not streamed yet), so the C2F cells of the second
 * substep hold the parent's state instead of populations streamed through
 * the shell without a collision.  MT_ITIME_EXTRAP explodes the second
 * substep from 1.5 fcol(t) - 0.5 fcol(t - 1) of the parent cells (t - 1:
 * the parent's previous step; the current values right after the state or
 * the option was set), the parent state at the half step to second order. */
int mt_case_set_interface_time(mt_ctx *ctx, int32_t case_id, int32_t mode);
/* Velocity of one face strategy (face 0..5 = West East South North Bot Top),
 * the input_v each nonEquilibrumExtrapolation_<face> / inlet strategy is
 * constructed with (NonEquilibrumExtrapolation.hpp:37-100; LBM_Manager.cpp:53-61
 * passes the same u0 to all six).  The face's boundary cells are reset to
 * f = fcol = feq(rho0, u), as D3Q19_BC_Strategy::initial_Feq does from the
 * velocity map (D3Q19_BC_Manager.hpp:157-167): boundary cells never collide,
 * so this is the velocity the fluid sees (a moving lid). */
int mt_case_set_face_velocity(mt_ctx *ctx, int32_t case_id, int32_t face, const double *u);

/* Lagrangian markers of a direct-forcing sphere (MT_IB_DF, no reference
 * counterpart; after mt_case_build).  ref[3][nm]: marker offsets from the
 * centre and dv[nm] their volume weights, in finest-level cells; center[3]
 * in finest-level cells; path[period][6]: the centre's displacement and
 * velocity at finest substep t (row t % period).  Each finest substep the
 * velocity at a marker is interpolated with the 3-point kernel of Roma,
 * Peskin & Berger, the force 2 rho (U - u) is spread back onto the
 * MT_SET_IB_BAND cells (exact int64 fixed-point sums), and the band cells
 * collide with Guo forcing; mt_get_force accumulates the force on the body. */
int mt_case_set_markers(mt_ctx *ctx, int32_t case_id, int64_t nm, const double *ref, const double *dv,
                        const double *center, int64_t period, const double *path);

/* ---- batches (no reference counterpart) --------------------------------
 * Independent multi-level cases stepped together: every substep of every
 * level runs one batched brick pass per model family (Q, collision, storage)
 * over all members that have that level, driven from a work list of their
 * 4x4x4 bricks; the members' other phases run on parallel graph branches.
 * A member level of 8192 bricks or more fills the GPU by itself and runs its
 * own brick pass on a branch beside the batched one.
 * Each coarse step of the batch is one captured CUDA graph (re-captured when
 * the membership changes).  A member ends every step in the state it would
 * reach stepped alone with MT_SCHED_FUSED (bit-identical: the same kernels
 * on the same cells).  Adding a case switches it to MT_SCHED_FUSED; a member
 * is stepped only through its batch (mt_step returns MT_ERR_STATE). */
int mt_batch_create(mt_ctx *ctx, int32_t *batch_id);
int mt_batch_destroy(mt_ctx *ctx, int32_t batch_id);
int mt_batch_add(mt_ctx *ctx, int32_t batch_id, int32_t case_id);
int mt_batch_remove(mt_ctx *ctx, int32_t batch_id, int32_t case_id);
int mt_batch_size(mt_ctx *ctx, int32_t batch_id, int32_t *n_cases);
/* n coarse steps of every member; asynchronous on the context stream */
int mt_batch_step(mt_ctx *ctx, int32_t batch_id, int32_t n_coarse_steps);
/* Admission helpers for a request loop (no reference counterpart): switch a
 * case to MT_SCHED_FUSED and build its fused-schedule tables (bricks, second
 * buffers, lookahead) now, synchronising only this context's stream; then
 * move the case to another context on the same device (a serving context
 * whose stream keeps running its batch meanwhile).  The case gets a new id
 * in dst; it must not be in a batch. */
int mt_case_prepare(mt_ctx *ctx, int32_t case_id);
int mt_case_transfer(mt_ctx *src, int32_t case_id, mt_ctx *dst, int32_t *new_id);
/* accumulated momentum-exchange force of treat() calls: fx, fy, fz, count
 * (LBM_Manager::accumIBForce, LBM_Manager.cpp:846-852) */
int mt_get_force(mt_ctx *ctx, int32_t case_id, double *out4);
int mt_reset_force(mt_ctx *ctx, int32_t case_id);

/* ---- asynchronous completion (no reference counterpart) ---------------
 * For a request loop that keeps a bounded number of steps in flight and
 * learns when a result is ready without synchronising the context.
 * mt_marker_record records the current point of the context stream and
 * returns its ticket (increasing from 0); mt_marker_done sets *done = 1 once
 * the stream has passed that point (it never blocks; recording blocks only
 * when 64 markers are outstanding).  mt_case_force_async enqueues a copy of
 * the accumulated force (as mt_get_force returns it) into page-locked memory
 * the case keeps; mt_case_force_copied returns that copy, which is complete
 * once a marker recorded after mt_case_force_async is done. */
int mt_marker_record(mt_ctx *ctx, int64_t *ticket);
int mt_marker_done(mt_ctx *ctx, int64_t ticket, int32_t *done);
int mt_case_force_async(mt_ctx *ctx, int32_t case_id);
int mt_case_force_copied(mt_ctx *ctx, int32_t case_id, double *out4);
/* The non-finite check of the state (mt_case_status's guard, over the
 * post-collision buffers every schedule steps from) that mt_case_force_async
 * also enqueues: MT_OK, or MT_ERR_NONFINITE when the copied flags show a NaN
 * or Inf population.  Valid under the same marker as the force copy.  The
 * reference stops on NaN by scanning on the host (LBM_Simulator.cpp:33-41). */
int mt_case_status_copied(mt_ctx *ctx, int32_t case_id);

#ifdef __cplusplus
}
#endif

#endif /* MT_LBM_H */
