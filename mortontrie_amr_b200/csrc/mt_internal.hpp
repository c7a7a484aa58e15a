// Internal types of libmtlbm: context, per-case device state, launch helpers.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/mt_lbm.h"
#include "mt_lattice.cuh"

namespace mt {

constexpr int kMaxLevels = MT_MAX_LEVELS;
constexpr int kNumSets = 6;  // lat_f, F2C, C2F, ghost C2F, ghost F2C, solid

// phases of the multi-level step (amr_phase): the reference's strategy calls,
// then the fused schedule's own passes
enum { PH_MACROS = 0, PH_COLLIDE, PH_STREAM, PH_EXPLOSION, PH_COALESCENCE, PH_BC, PH_IB, PH_BC_INOUT,
       PH_BC_FACE0 = 8, PH_F2C_COLLIDE = 16, PH_PULL_COLLIDE, PH_PRIME, PH_COAL_COLLIDE,
       PH_SYNC_F, PH_DF, PH_BAND_GRID, PH_FACE_EQ0 = 24, PH_BC_HH = 32, PH_EXPLOSION_B, PH_EXPL_SAVE };

// per-cell tag bits (which reference index sets the cell belongs to)
enum : uint32_t {
    TAG_LATF = 1u,
    TAG_F2C = 2u,
    TAG_C2F = 4u,
    TAG_GC2F = 8u,
    TAG_GF2C = 16u,
    TAG_BC = 32u,
    TAG_SF = 64u,
    TAG_IB = 128u,
    TAG_BAND = 256u,  // direct-forcing band
};

// device error flags raised by build / step kernels
enum : int {
    DEVERR_MISSING_CHILD = 1,     // a child of an interface cell is not stored (the reference's .at() throws)
    DEVERR_MISSING_BC_NBR = 2,    // a boundary cell's reserved neighbour is not stored
    DEVERR_DIS_NOT_FINEST = 4,    // a dis key is not a finest-level cell
    DEVERR_NONFINITE = 8,         // NaN/Inf population found by the guard
};

struct Level {
    int64_t n = 0;
    uint64_t *key = nullptr;   // sorted unique Morton keys
    uint32_t *tag = nullptr;
    int8_t *bcidx = nullptr;   // lat_bc index or -1
    int32_t *disrow = nullptr; // row in the dis table or -1
    int32_t *nbr = nullptr;    // [(Q-1) * n]: index of the cell at key + e_k (k >= 1) or -1
    void *f = nullptr, *fcol = nullptr;  // [Q * n] populations in the case's storage type
    // fused schedule: the second post-collision buffer (the next substep's fcol,
    // swapped with fcol at each substep) and the lat_f cells it collides (IB
    // cells of the finest level excluded, they have their own kernel)
    void *fcol_alt = nullptr;
    int32_t *fused_list = nullptr; int64_t nfused = 0;
    // 4x4x4 Morton bricks of the level's key set (fused schedule): a brick's
    // cells are contiguous in key order, so a cell at local Morton index m is
    // stored iff bit m of the brick's mask is set, at index
    // start + popcount(mask & (2^m - 1)).  bnbr[27 * b + s] is the brick at
    // offset (s % 3 - 1, s / 3 % 3 - 1, s / 9 - 1) or -1; bhalo resolves them per
    // position of the 6x6x6 neighbourhood; bcls[64 * b + m] is
    // the cell's work in the fused pass (0 none, 1 stream + collide, 2 stream + copy).
    bool bricks = false;
    int brick_variant = 0;  // fused brick pass: 0 one cell per lane step, 1 two cells with packed FP32 pairs, 2 one cell with more registers, 3 both cells unrolled
    int64_t nbrick = 0;
    int32_t *bstart = nullptr;
    uint64_t *bmask = nullptr;
    int32_t *bnbr = nullptr;
    uint8_t *bcls = nullptr;
    int32_t *bhalo = nullptr;  // [216 * b]: cell index at each position of the brick's 6x6x6 neighbourhood, or -1
    void *rho = nullptr, *u = nullptr;   // [n], [3 * n] macroscopic fields (double, or float for reduced storage)
    int32_t *list[kNumSets] = {};
    int64_t nlist[kNumSets] = {};
    int32_t *collide_list = nullptr; int64_t ncollide = 0;  // lat_f then F2C
    int32_t *stream_list = nullptr;  int64_t nstream = 0;   // lat_f then C2F
    int32_t *bclist[26] = {};
    int64_t nbc[26] = {};
    int32_t *iblist = nullptr; int64_t nib = 0;             // finest lat_f cells with dis rows
    int32_t *band = nullptr; int64_t nband = 0;             // direct-forcing band (finest level)
    int32_t *collide_nb = nullptr; int64_t ncollide_nb = 0; // lat_f (not band) then F2C
    // explosion sources on the parent level (F2C then ghost F2C) and their children on this level
    int32_t *expl_src = nullptr; int32_t *expl_child = nullptr; int64_t nexpl = 0, nexpl_f2c = 0;
    void *expl_prev = nullptr;  // MT_ITIME_EXTRAP: [Q * nexpl] the sources' parent values at the parent's previous step
    double *info_prev = nullptr;  // mt_case_info: [3][nlist[0]] the lat_f velocities the last call saw
    bool info_have = false;
    // coalescence: F2C cells of this level and their children on the next level
    int32_t *coal_child = nullptr;
    // raw uploads, consumed by the build
    std::vector<uint64_t> raw_keys;
    std::vector<uint8_t> raw_set;  // 0..5 sets, 16 + b for lat_bc[b]
    // the same pairs generated on the device (mt_case_generate), used instead
    uint64_t *draw_keys = nullptr;
    uint8_t *draw_set = nullptr;
    int64_t ndraw = 0;
};

// one case level in a batched brick pass
struct BrickSlot {
    const int32_t *halo = nullptr;
    const uint8_t *cls = nullptr;
    const void *fcol = nullptr;  // current post-collision buffer
    void *f = nullptr, *fnext = nullptr, *rho = nullptr, *u = nullptr;
    long long *acc = nullptr;  // direct-forcing accumulator: band macros in the pass (finest level), else null
    double tau = 1.0;
    uint32_t n = 0;
    int32_t textbook = 0, fall = 0, macros = 0;
};
constexpr int kMaxBatchSlots = 128;
// a member level with at least this many bricks fills the GPU by itself: it
// runs its own brick pass (same kernel as alone) beside the batched one
constexpr int64_t kBatchOwnBricks = 8192;
// a batched brick pass: slots and the prefix offsets of their bricks
struct BrickBatch {
    int32_t nslots = 0;
    int32_t pad = 0;
    int64_t total = 0;
    int64_t off[kMaxBatchSlots + 1] = {};
    BrickSlot slot[kMaxBatchSlots];
};

struct Case {
    mt_case_desc d{};
    bool dense = false;
    bool built = false;
    Level lv[kMaxLevels];
    int64_t ndis = 0;
    uint64_t *dis_key = nullptr;
    double *dis = nullptr;
    std::vector<uint64_t> h_dis_key;
    std::vector<double> h_dis;
    bool dis_on_device = false;  // dis_key / dis generated on the device (ndis set)
    std::vector<double> h_tri;   // solid surface triangles [n][3][3], coarse-cell units (mt_case_set_surface)
    // refinement regions (mt_case_set_region): h_reg[l] the level-(l-1)
    // cells refined to level l, a dense mask over [reg_lo[l], reg_lo[l] + reg_n[l])
    std::vector<uint8_t> h_reg[MT_MAX_LEVELS + 1];
    int64_t reg_lo[MT_MAX_LEVELS + 1][3] = {};
    int64_t reg_n[MT_MAX_LEVELS + 1][3] = {};
    double *ib_force = nullptr;  // [3 * nib] per-cell force of the last treat()
    double *force_acc = nullptr; // [4] fx, fy, fz, treat count
    double *h_force = nullptr;   // [6] page-locked: force_acc copy [4], then the guard flags (int) (mt_case_force_async)
    int *dev_err = nullptr;
    MortonGeom geom{};
    // dense uniform path
    int bits = 0;        // log2 of the cube edge
    int64_t N = 0;       // cells
    void *A = nullptr, *B = nullptr;  // populations [Q * N] in the storage type
    bool a_is_fcol = false;           // false: A holds post-stream f; true: A holds post-collision fcol
    double *bc_tmp = nullptr;         // scratch of the boundary sweep (per set)
    // every boundary set at once: cells, their set, scratch [18][n]
    int32_t *bc_all = nullptr;
    int8_t *bc_setb = nullptr;
    double *bc_tmp_all = nullptr;
    int64_t nbc_all = 0;
    int dense_block = 256;            // threads per block of the fused kernel (autotuned)
    // captured coarse step of the phase schedule (recorded with level 0's
    // post-collision buffer in parity graph_par0)
    cudaGraphExec_t graph = nullptr;
    int64_t graph_launches = 0;
    int graph_par0 = 0;
    // fused schedule: one graph per parity of level 0's buffers (levels >= 1
    // swap an even number of times per coarse step), and whether the
    // lookahead buffers hold the collision of the current f
    int schedule = MT_SCHED_PHASES;
    int scaling = MT_SCALE_REFERENCE;  // interface rescaling of the non-equilibrium part
    int itime = MT_ITIME_REFERENCE;    // substeps in which a fine level explodes from its parent
    bool prev_stale = true;            // expl_prev no longer belongs to the state (MT_ITIME_EXTRAP)
    Shift shift[kMaxLevels];  // per level: storage shift of the reduced storages (from d.u_shift)
    double face_u[6][3] = {};          // bc_velocity of each face's strategy (u_bc unless set)
    // direct-forcing markers (MT_IB_DF)
    int64_t nm = 0;
    double *mref = nullptr, *mdv = nullptr, *path = nullptr, *mforce = nullptr;
    double center[3] = {0, 0, 0};
    int64_t period = 1;
    long long *tstep = nullptr;
    int64_t coarse_steps = 0;  // coarse steps taken through mt_step / mt_batch_step (mt_case_get_step)
    long long *acc = nullptr;  // [3][n_L] Eulerian force, fixed point
    // dense index of the band cells over the box the markers' stencils can reach
    int32_t *mgrid = nullptr;
    int64_t mlo[3] = {0, 0, 0}, mdim[3] = {0, 0, 0};
    bool use_bricks = true;  // fused pass over 4x4x4 bricks where a level allows it (else cell lists)
    bool primed = false;
    int par0 = 0;
    cudaGraphExec_t fgraph[2] = {nullptr, nullptr};
    int64_t fgraph_launches[2] = {0, 0};
    // second stream of the fused schedule: the IB cells' treat + collision
    // overlaps the finest level's fused pass (disjoint cells)
    int macros_now = 0;  // set while recording a level's last substep of the coarse step
    int pull_mode = 0;   // PH_PULL_COLLIDE: 0 every cell, 1 the IB cells only (a batch runs the bricks)
    bool no_side = false; // IB on the calling stream (batch recording)
    int in_batch = 0;     // batches holding the case
    bool f_stale = false; // fused passes left class-1 brick cells' streamed f unstored (amr_sync_f)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
};

// Cases stepped together (mt_batch_*): one batched brick pass per level,
// substep and model family over all of them, their other phases on parallel
// graph branches.  Level 0 of every member swaps buffers once per coarse
// step, so two captured graphs alternate (par).
struct Batch {
    std::vector<int32_t> ids;
    // [0], [1]: one coarse step from level-0 parity 0 / 1; [2]: two coarse
    // steps (back to the same parity, valid from either)
    cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
    int64_t graph_launches[3] = {0, 0, 0};
    BrickBatch *ddesc[3] = {nullptr, nullptr, nullptr};
    std::vector<BrickBatch> hdesc[3];  // host copies (kept alive for the asynchronous upload)
    int par = 0;
    std::vector<cudaStream_t> pool;
    std::vector<cudaEvent_t> ev_join;
    cudaEvent_t ev_fork = nullptr;
    cudaStream_t free_stream = nullptr;  // the stream the batch last ran on
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<Case *> cases;
    std::vector<Batch *> batches;
    std::string last_error;
    int64_t launches = 0;  // kernels this library launched (graph nodes count per replay)
    // stream markers (mt_marker_record): a ring of events, slot = ticket % size
    std::vector<cudaEvent_t> markers;
    int64_t next_marker = 0;
};
constexpr int kMarkerRing = 64;

// kernel launchers implemented in the .cu files
int amr_build(Ctx &ctx, Case &c);
// device lattice classification: raw sets of every level and the dis table
int amr_generate(Ctx &ctx, Case &c, const mt_mesh_spec &spec);
// the state of src carried onto dst's lattice (counts: [4 * level + kind] or null)
int amr_remap(Ctx &ctx, Case &dst, Case &src, int64_t *counts);
int amr_init_equilibrium(Ctx &ctx, Case &c, double rho0, const double *u0);
int amr_lbm_kernel(Ctx &ctx, Case &c, int level);
int amr_step(Ctx &ctx, Case &c, int n);
int amr_phase(Ctx &ctx, Case &c, int phase, int level);
int amr_find(Ctx &ctx, Case &c, int level, const uint64_t *h_keys, int64_t n, int64_t *h_idx);
int amr_guard(Ctx &ctx, Case &c, int *flags);
int amr_get(Ctx &ctx, Case &c, int level, double *h_f, double *h_fcol);
int amr_set(Ctx &ctx, Case &c, int level, const double *h_f, const double *h_fcol);
int amr_macros(Ctx &ctx, Case &c, int level, double *h_rho, double *h_u);
int amr_reduce(Ctx &ctx, Case &c, double *h_out);
int amr_sync_f(Ctx &ctx, Case &c);
int amr_info(Ctx &ctx, Case &c, double *h_out);
// MT_ITIME_EXTRAP: saved explosion sources allocated and, when stale, taken from the state
int amr_prev_sync(Ctx &ctx, Case &c);
int amr_set_face(Ctx &ctx, Case &c, int face, const double *u);
int amr_prime(Ctx &ctx, Case &c);
int batch_step(Ctx &ctx, Batch &b, const std::vector<Case *> &cases, int n);
void batch_drop(Batch &b);
void batch_free(Batch &b);

// multi-level phases, one explicit instantiation per storage type
// (mt_amr_f64.cu builds the FP64 one without FMA contraction)
template <class S> struct AmrOps {
    static int phase(Ctx &ctx, Case &c, int phase, int level);
    static int upload_tables(Ctx &ctx);
    static int alloc(Ctx &ctx, Case &c, int level);
    static int init_eq(Ctx &ctx, Case &c, double rho0, const double *u0);
    static int get(Ctx &ctx, Case &c, int level, int which, double *d_out);      // which: 0 f, 1 fcol
    static int set(Ctx &ctx, Case &c, int level, int which, const double *d_in);
    static int macros_out(Ctx &ctx, Case &c, int level, double *d_rho, double *d_u);
    // non-finite populations into c.dev_err; current_only: the post-collision
    // buffers alone (the state every schedule steps from), no f rebuild needed
    static int guard(Ctx &ctx, Case &c, bool current_only = false);
    // FP64 mass, momentum, kinetic energy per level over the collide list and
    // the volume-weighted total: d_out[(max_level + 2) * 5]
    static int reduce(Ctx &ctx, Case &c, double *d_out);
    // time every form of every brick level's fused pass (into scratch, state
    // untouched) and keep the fastest in Level::brick_variant;
    // ms[MT_BRICK_FORMS * level + form], variant[level] (-1: no brick pass on the level)
    static int tune_bricks(Ctx &ctx, Case &c, int32_t *variant, float *ms);
    // infoPrint's diagnostics per level into d_out [(max_level + 1) * 4]
    // (mt_case_info)
    static int info(Ctx &ctx, Case &c, double *d_out);
    // batched brick pass (descriptor in device memory, total bricks known on the host)
    static int batch_pass(Ctx &ctx, int q, int coll, const BrickBatch *d_desc, int64_t total, const Shift &sh);
    // src's state carried onto dst's lattice (same Q, levels, storage)
    static int remap(Ctx &ctx, Case &dst, Case &src, int64_t *counts);
};
void amr_free(Case &c);
// forget the fused schedule's graphs and brick tables (rebuilt at the next fused step)
void amr_drop_fused(Case &c);

// dense uniform path, one explicit instantiation per storage type
// (mt_dense_f64.cu builds the FP64 one without FMA contraction)
template <class S> struct DenseOps {
    static int step(Ctx &ctx, Case &c, int mode);  // mode: 0 fused pull+collide, 1 collide in place
    static int init(Ctx &ctx, Case &c, const double *rho, const double *ux, const double *uy, const double *uz,
                    double rho0, const double *u0);
    static int get(Ctx &ctx, Case &c, double *d_f, int pull);
    static int set(Ctx &ctx, Case &c, const double *d_f);
    static int macros(Ctx &ctx, Case &c, double *d_rho, double *d_u);
    static int reduce(Ctx &ctx, Case &c, double *d_out);
    // the same two launches as reduce() into caller-provided device scratch:
    // partial[5 * ceil(N / 256)] per-block sums and d_out[5] totals; allocates nothing
    static int reduce_into(Ctx &ctx, Case &c, double *partial, double *d_out);
    // time the fused kernel at each candidate block size (A -> B, no swap:
    // the state is untouched) and keep the fastest in c.dense_block
    static int tune(Ctx &ctx, Case &c, float *ms_out, int *blocks_out, int *n_out);
};

// call fn with a null pointer of the multi-level case's storage type
template <class F> int amr_dispatch(Case &c, F &&fn)
{
    switch (c.d.storage) {
    case MT_STORE_F64: return fn((double *)nullptr);
    case MT_STORE_F32: return fn((float *)nullptr);
    case MT_STORE_F16: return fn((__half *)nullptr);
    default: return fn((__nv_bfloat16 *)nullptr);
    }
}

// error helpers
int set_err(Ctx &ctx, int code, const std::string &msg);
#define MT_CUDA(ctx, call)                                                                          \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return ::mt::set_err((ctx), MT_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)
#define MT_LAUNCHED(ctx)                                                                            \
    do {                                                                                            \
        cudaError_t e_ = cudaGetLastError();                                                        \
        if (e_ != cudaSuccess)                                                                      \
            return ::mt::set_err((ctx), MT_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
        (ctx).launches++;                                                                           \
    } while (0)

inline unsigned grid_for(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }

}  // namespace mt
