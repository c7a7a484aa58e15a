// C ABI of libmtlbm (declarations and reference citations in include/mt_lbm.h).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>

#include "mt_internal.hpp"

extern template struct mt::DenseOps<double>;
extern template struct mt::DenseOps<float>;
extern template struct mt::DenseOps<__half>;
extern template struct mt::DenseOps<__nv_bfloat16>;

struct mt_ctx {
    mt::Ctx c;
};

namespace mt {

int set_err(Ctx &ctx, int code, const std::string &msg)
{
    ctx.last_error = msg;
    return code;
}

namespace {


int get_case(mt_ctx *h, int32_t id, Case **out)
{
    if (!h) return MT_ERR_ARG;
    Ctx &ctx = h->c;
    if (id < 0 || id >= (int32_t)ctx.cases.size() || !ctx.cases[id])
        return set_err(ctx, MT_ERR_ARG, "unknown case id");
    *out = ctx.cases[id];
    return MT_OK;
}

int check_desc(Ctx &ctx, const mt_case_desc *d)
{
    if (!d) return set_err(ctx, MT_ERR_ARG, "null case description");
    if (d->q != 19 && d->q != 27) return set_err(ctx, MT_ERR_ARG, "q must be 19 or 27");
    if (d->max_level < 0 || d->max_level >= MT_MAX_LEVELS) return set_err(ctx, MT_ERR_ARG, "max_level out of range");
    if (d->collision != MT_COLL_LBGK && d->collision != MT_COLL_CUMULANT)
        return set_err(ctx, MT_ERR_ARG, "unknown collision model");
    if (d->collision == MT_COLL_CUMULANT && d->q != 27)
        return set_err(ctx, MT_ERR_ARG, "the cumulant collision needs D3Q27");
    if (d->storage < MT_STORE_F64 || d->storage > MT_STORE_BF16) return set_err(ctx, MT_ERR_ARG, "unknown storage");
    if (d->ib_method != MT_IB_DW && d->ib_method != MT_IB_FH && d->ib_method != MT_IB_DF)
        return set_err(ctx, MT_ERR_ARG, "unknown immersed-boundary method");
    if (d->bc_mode != MT_BC_NEQ && d->bc_mode != MT_BC_ZOUHE_OUTFLOW && d->bc_mode != MT_BC_ZOUHE_HH)
        return set_err(ctx, MT_ERR_ARG, "unknown boundary mode");
    if (d->bc_mode == MT_BC_ZOUHE_HH && (d->q != 19 || d->collision != MT_COLL_LBGK))
        return set_err(ctx, MT_ERR_ARG, "the Zou-He / Hecht-Harting boundary is D3Q19 LBGK");
    if (d->ib_method == MT_IB_DF && d->collision != MT_COLL_LBGK)
        return set_err(ctx, MT_ERR_ARG, "direct forcing is implemented with the LBGK collision");
    for (int l = 0; l <= d->max_level; ++l)
        if (!(d->tau[l] > 0.5)) return set_err(ctx, MT_ERR_ARG, "tau must exceed 1/2 on every level");
    for (int a = 0; a < 3; ++a)
        if (d->extent0[a] <= 0 || d->extent0[a] > ((int64_t)1 << (21 - d->max_level)))
            return set_err(ctx, MT_ERR_ARG, "extent does not fit the 21-bit Morton coordinate");
    for (int l = 0; l < MT_MAX_LEVELS; ++l)
        for (int a = 0; a < 3; ++a)
            if (!(std::fabs(d->u_shift[l][a]) <= 0.5))
                return set_err(ctx, MT_ERR_ARG, "u_shift must be finite with |u_s| <= 0.5 per axis");
    return MT_OK;
}

int add_case(Ctx &ctx, Case *c, int32_t *id)
{
    ctx.cases.push_back(c);
    *id = (int32_t)ctx.cases.size() - 1;
    return MT_OK;
}

template <class F> int dense_dispatch(Case &c, F &&fn)
{
    switch (c.d.storage) {
    case MT_STORE_F64: return fn((double *)nullptr);
    case MT_STORE_F32: return fn((float *)nullptr);
    case MT_STORE_F16: return fn((__half *)nullptr);
    default: return fn((__nv_bfloat16 *)nullptr);
    }
}

size_t storage_bytes(int s) { return s == MT_STORE_F64 ? 8 : (s == MT_STORE_F32 ? 4 : 2); }

int phase_call(mt_ctx *h, int32_t id, int phase, int level)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    if (c->dense) return set_err(h->c, MT_ERR_STATE, "per-phase calls need a multi-level case (use mt_step)");
    if (!c->built) return set_err(h->c, MT_ERR_STATE, "case not built");
    if ((rc = amr_prev_sync(h->c, *c))) return rc;
    if ((rc = amr_sync_f(h->c, *c))) return rc;
    c->primed = false;  // the fused schedule's lookahead no longer matches f
    return amr_phase(h->c, *c, phase, level);
}

}  // namespace
}  // namespace mt

using namespace mt;

extern "C" {

int mt_create(int32_t device, mt_ctx **out)
{
    if (!out) return MT_ERR_ARG;
    *out = nullptr;
    mt_ctx *h = new (std::nothrow) mt_ctx();
    if (!h) return MT_ERR_ARG;
    h->c.device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->c.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return MT_ERR_CUDA;
    }
    h->c.own_stream = true;
    // stream-ordered allocations of case builds and re-meshes keep their
    // memory in the device's pool between builds instead of returning it at
    // every synchronisation (re-mapping it costs more than the build)
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    *out = h;
    return MT_OK;
}

int mt_destroy(mt_ctx *h)
{
    if (!h) return MT_ERR_ARG;
    cudaSetDevice(h->c.device);
    cudaStreamSynchronize(h->c.stream);
    for (Batch *b : h->c.batches)
        if (b) {
            batch_free(*b);
            delete b;
        }
    for (Case *c : h->c.cases)
        if (c) {
            amr_free(*c);
            if (c->A) cudaFree(c->A);
            if (c->B) cudaFree(c->B);
            delete c;
        }
    for (cudaEvent_t e : h->c.markers)
        if (e) cudaEventDestroy(e);
    if (h->c.own_stream) cudaStreamDestroy(h->c.stream);
    delete h;
    return MT_OK;
}

int mt_set_priority(mt_ctx *h, int32_t high)
{
    if (!h) return MT_ERR_ARG;
    Ctx &ctx = h->c;
    if (!ctx.own_stream) return set_err(ctx, MT_ERR_STATE, "the context runs on a caller's stream");
    MT_CUDA(ctx, cudaSetDevice(ctx.device));
    int lo = 0, hi = 0;
    MT_CUDA(ctx, cudaDeviceGetStreamPriorityRange(&lo, &hi));
    cudaStream_t s = nullptr;
    MT_CUDA(ctx, cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, high ? hi : lo));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    cudaStreamDestroy(ctx.stream);
    ctx.stream = s;
    return MT_OK;
}

int mt_marker_record(mt_ctx *h, int64_t *ticket)
{
    if (!h || !ticket) return MT_ERR_ARG;
    Ctx &ctx = h->c;
    MT_CUDA(ctx, cudaSetDevice(ctx.device));
    if (ctx.markers.empty()) {
        ctx.markers.assign(kMarkerRing, nullptr);
        for (auto &e : ctx.markers) MT_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const int64_t t = ctx.next_marker;
    cudaEvent_t e = ctx.markers[t % kMarkerRing];
    // the slot's previous marker must have passed before the slot is reused,
    // so that a ticket older than the ring is known to be done
    if (t >= kMarkerRing) MT_CUDA(ctx, cudaEventSynchronize(e));
    MT_CUDA(ctx, cudaEventRecord(e, ctx.stream));
    ctx.next_marker = t + 1;
    *ticket = t;
    return MT_OK;
}

int mt_marker_done(mt_ctx *h, int64_t ticket, int32_t *done)
{
    if (!h || !done) return MT_ERR_ARG;
    Ctx &ctx = h->c;
    if (ticket < 0 || ticket >= ctx.next_marker) return set_err(ctx, MT_ERR_ARG, "unknown marker ticket");
    if (ticket < ctx.next_marker - kMarkerRing) {
        *done = 1;
        return MT_OK;
    }
    const cudaError_t e = cudaEventQuery(ctx.markers[ticket % kMarkerRing]);
    if (e == cudaSuccess) {
        *done = 1;
    } else if (e == cudaErrorNotReady) {
        cudaGetLastError();
        *done = 0;
    } else {
        return set_err(ctx, MT_ERR_CUDA, std::string("cudaEventQuery: ") + cudaGetErrorString(e));
    }
    return MT_OK;
}

const char *mt_last_error(const mt_ctx *h) { return h ? h->c.last_error.c_str() : "null context"; }

int mt_set_stream(mt_ctx *h, void *stream)
{
    if (!h) return MT_ERR_ARG;
    Ctx &ctx = h->c;
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    if (ctx.own_stream) cudaStreamDestroy(ctx.stream);
    if (stream) {
        ctx.stream = (cudaStream_t)stream;
        ctx.own_stream = false;
    } else {
        MT_CUDA(ctx, cudaStreamCreateWithFlags(&ctx.stream, cudaStreamNonBlocking));
        ctx.own_stream = true;
    }
    // captured graphs are launched on whatever stream is current; nothing to redo
    return MT_OK;
}

int mt_synchronize(mt_ctx *h)
{
    if (!h) return MT_ERR_ARG;
    MT_CUDA(h->c, cudaStreamSynchronize(h->c.stream));
    return MT_OK;
}

int mt_launch_count(const mt_ctx *h, int64_t *out)
{
    if (!h || !out) return MT_ERR_ARG;
    *out = h->c.launches;
    return MT_OK;
}

int mt_case_create(mt_ctx *h, const mt_case_desc *d, int32_t *id)
{
    if (!h || !id) return MT_ERR_ARG;
    Ctx &ctx = h->c;
    int rc = check_desc(ctx, d);
    if (rc) return rc;
    Case *c = new Case();
    c->d = *d;
    for (int l = 0; l < MT_MAX_LEVELS; ++l) c->shift[l] = make_shift(d->q, d->u_shift[l]);
    return add_case(ctx, c, id);
}

int mt_case_create_dense(mt_ctx *h, const mt_case_desc *d, int32_t *id)
{
    if (!h || !id) return MT_ERR_ARG;
    Ctx &ctx = h->c;
    int rc = check_desc(ctx, d);
    if (rc) return rc;
    if (d->max_level != 0) return set_err(ctx, MT_ERR_ARG, "the dense path has one level");
    if (!d->periodic[0] || !d->periodic[1] || !d->periodic[2])
        return set_err(ctx, MT_ERR_ARG, "the dense path is periodic on every axis");
    const int64_t e = d->extent0[0];
    if (e != d->extent0[1] || e != d->extent0[2] || (e & (e - 1)) != 0 || e < 2 || e > 1024)
        return set_err(ctx, MT_ERR_ARG, "the dense path needs a cube of 2^b cells per edge, 2 <= 2^b <= 1024");
    // every level's shift is checked, not only level 0's: a shift requested
    // for any level would otherwise be dropped without a word
    for (int l = 0; l < MT_MAX_LEVELS; ++l)
        for (int a = 0; a < 3; ++a)
            if (d->u_shift[l][a] != 0.0)
                return set_err(ctx, MT_ERR_ARG, "the dense path stores f - w (u_shift must be zero on every level)");
    Case *c = new Case();
    c->d = *d;
    c->dense = true;
    int bits = 0;
    while (((int64_t)1 << bits) < e) ++bits;
    c->bits = bits;
    c->N = e * e * e;
    const size_t bytes = storage_bytes(d->storage) * (size_t)d->q * (size_t)c->N;
    cudaError_t ea = cudaMalloc(&c->A, bytes);
    cudaError_t eb = ea == cudaSuccess ? cudaMalloc(&c->B, bytes) : ea;
    if (eb != cudaSuccess) {
        if (c->A) cudaFree(c->A);
        delete c;
        return set_err(ctx, MT_ERR_CUDA, std::string("dense allocation: ") + cudaGetErrorString(eb));
    }
    c->built = true;
    rc = add_case(ctx, c, id);
    if (rc) return rc;
    const double u0[3] = {d->u_bc[0], d->u_bc[1], d->u_bc[2]};
    return dense_dispatch(*c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return DenseOps<S>::init(ctx, *c, nullptr, nullptr, nullptr, nullptr, d->rho0, u0);
    });
}

int mt_case_destroy(mt_ctx *h, int32_t id)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    cudaStreamSynchronize(h->c.stream);
    // leave every batch that holds the case
    for (Batch *b : h->c.batches)
        if (b)
            for (size_t k = 0; k < b->ids.size(); ++k)
                if (b->ids[k] == id) {
                    b->ids.erase(b->ids.begin() + k);
                    batch_drop(*b);
                    break;
                }
    amr_free(*c);
    if (c->A) cudaFree(c->A);
    if (c->B) cudaFree(c->B);
    delete c;
    h->c.cases[id] = nullptr;
    return MT_OK;
}

int mt_case_add_set(mt_ctx *h, int32_t id, int32_t level, int32_t set_id, const uint64_t *keys, int64_t n)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || c->built) return set_err(ctx, MT_ERR_STATE, "sets can only be added before the build");
    if (level < 0 || level > c->d.max_level) return set_err(ctx, MT_ERR_ARG, "level out of range");
    if (n < 0 || (n > 0 && !keys)) return set_err(ctx, MT_ERR_ARG, "bad key array");
    uint8_t s;
    if (set_id >= MT_SET_LAT_BC0 && set_id < MT_SET_LAT_BC0 + 26) {
        if (level != 0) return set_err(ctx, MT_ERR_ARG, "boundary sets live on level 0");
        s = (uint8_t)(16 + set_id - MT_SET_LAT_BC0);
    } else if (set_id >= 0 && set_id < kNumSets) {
        s = (uint8_t)set_id;
    } else if (set_id == MT_SET_IB_BAND) {
        if (level != c->d.max_level) return set_err(ctx, MT_ERR_ARG, "the forcing band lives on the finest level");
        s = (uint8_t)MT_SET_IB_BAND;
    } else {
        return set_err(ctx, MT_ERR_ARG, "unknown set id");
    }
    Level &lv = c->lv[level];
    lv.raw_keys.insert(lv.raw_keys.end(), keys, keys + n);
    lv.raw_set.insert(lv.raw_set.end(), (size_t)n, s);
    return MT_OK;
}

int mt_case_set_dis(mt_ctx *h, int32_t id, const uint64_t *keys, const double *rows, int64_t n)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || c->built) return set_err(ctx, MT_ERR_STATE, "dis can only be set before the build");
    if (n < 0 || (n > 0 && (!keys || !rows))) return set_err(ctx, MT_ERR_ARG, "bad dis arrays");
    for (int64_t i = 1; i < n; ++i)
        if (keys[i] <= keys[i - 1]) return set_err(ctx, MT_ERR_ARG, "dis keys must be strictly ascending");
    c->h_dis_key.assign(keys, keys + n);
    c->h_dis.assign(rows, rows + n * (c->d.q - 1));
    return MT_OK;
}

int mt_case_build(mt_ctx *h, int32_t id)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || c->built) return set_err(ctx, MT_ERR_STATE, "case already built");
    MT_CUDA(ctx, cudaSetDevice(ctx.device));
    rc = amr_build(ctx, *c);
    if (rc) return rc;
    const double u0[3] = {c->d.u_bc[0], c->d.u_bc[1], c->d.u_bc[2]};
    rc = amr_init_equilibrium(ctx, *c, c->d.rho0, u0);
    if (rc) return rc;
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}

int mt_case_set_surface(mt_ctx *h, int32_t id, const double *tri, int64_t n)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || c->built) return set_err(ctx, MT_ERR_STATE, "the surface can only be set before the build");
    if (n < 0 || (n > 0 && !tri) || n > INT32_MAX) return set_err(ctx, MT_ERR_ARG, "bad triangle array");
    for (int64_t i = 0; i < 9 * n; ++i)
        if (!std::isfinite(tri[i])) return set_err(ctx, MT_ERR_ARG, "non-finite triangle vertex");
    c->h_tri.assign(tri, tri + 9 * n);
    return MT_OK;
}

int mt_case_set_region(mt_ctx *h, int32_t id, int32_t level, const int64_t *lo, const int64_t *shape,
                       const uint8_t *mask)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || c->built) return set_err(ctx, MT_ERR_STATE, "a region can only be set before the build");
    if (level < 1 || level > c->d.max_level) return set_err(ctx, MT_ERR_ARG, "region level out of range");
    if (!lo || !shape || !mask) return set_err(ctx, MT_ERR_ARG, "null region argument");
    int64_t n = 1;
    for (int a = 0; a < 3; ++a) {
        const int64_t ext = c->d.extent0[a] << (level - 1);
        if (shape[a] < 1 || lo[a] < 0 || lo[a] + shape[a] > ext)
            return set_err(ctx, MT_ERR_ARG, "region box outside the coarser level's extent");
        n *= shape[a];
        if (n > INT32_MAX) return set_err(ctx, MT_ERR_ARG, "a region box above 2^31 cells");
    }
    c->h_reg[level].assign(mask, mask + n);
    for (int a = 0; a < 3; ++a) {
        c->reg_lo[level][a] = lo[a];
        c->reg_n[level][a] = shape[a];
    }
    return MT_OK;
}

int mt_case_generate(mt_ctx *h, int32_t id, const mt_mesh_spec *sp)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || c->built) return set_err(ctx, MT_ERR_STATE, "case already built");
    if (!sp) return set_err(ctx, MT_ERR_ARG, "null mesh spec");
    for (int l = 0; l <= c->d.max_level; ++l)
        if (!c->lv[l].raw_keys.empty()) return set_err(ctx, MT_ERR_STATE, "sets were already added to the case");
    if (!c->h_dis_key.empty()) return set_err(ctx, MT_ERR_STATE, "dis was already set");
    const int L = c->d.max_level;
    for (int a = 0; a < 3; ++a) {
        if (sp->coarse[a] != c->d.extent0[a]) return set_err(ctx, MT_ERR_ARG, "spec extent differs from the case's");
        if ((sp->boundary_bc[a] != 0) == (c->d.periodic[a] != 0))
            return set_err(ctx, MT_ERR_ARG, "spec boundary differs from the case's periodic axes");
        if (sp->coarse[a] < 1 || (sp->coarse[a] << L) > (int64_t(1) << 21))
            return set_err(ctx, MT_ERR_ARG, "extent out of the 21-bit Morton range");
    }
    if (sp->sphere < 0 || sp->sphere > 3) return set_err(ctx, MT_ERR_ARG, "sphere must be 0, 1, 2 or 3");
    if (sp->sphere == 2 && c->d.ib_method != MT_IB_DF)
        return set_err(ctx, MT_ERR_ARG, "a forcing band needs ib_method MT_IB_DF");
    if ((sp->sphere == 1 || sp->sphere == 2) && !(sp->radius > 0.0))
        return set_err(ctx, MT_ERR_ARG, "sphere radius must be positive");
    if (sp->sphere == 3 && c->h_tri.empty()) return set_err(ctx, MT_ERR_STATE, "no surface set (mt_case_set_surface)");
    bool regions = false;
    for (int l = 0; l < L; ++l) {
        if (sp->has_refine[l] < 0 || sp->has_refine[l] > 2) return set_err(ctx, MT_ERR_ARG, "has_refine must be 0, 1 or 2");
        regions |= sp->has_refine[l] == 2;
    }
    if (regions)
        for (int l = 0; l < L; ++l) {
            if (sp->has_refine[l] != 2)
                return set_err(ctx, MT_ERR_ARG, "regions refine every level or none (no boxes beside them)");
            if (c->h_reg[l + 1].empty()) return set_err(ctx, MT_ERR_STATE, "no region set for a refined level");
        }
    {
        int64_t lo[3] = {0, 0, 0}, hi[3] = {sp->coarse[0], sp->coarse[1], sp->coarse[2]};
        for (int l = 0; l < L; ++l) {
            if (!sp->has_refine[l]) break;
            for (int a = 0; a < 3; ++a) {
                // the refined cells in level-l cells: the box, or the region's box
                const int64_t rl = regions ? c->reg_lo[l + 1][a] : sp->refine_lo[l][a];
                const int64_t rh = regions ? c->reg_lo[l + 1][a] + c->reg_n[l + 1][a] : sp->refine_hi[l][a];
                if (rl < lo[a] || rh > hi[a] || rh - rl < 1)
                    return set_err(ctx, MT_ERR_ARG, regions ? "refinement region outside its level's domain"
                                                            : "refinement box outside its level's domain");
                lo[a] = 2 * rl;
                hi[a] = 2 * rh;
            }
            if ((hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]) > INT32_MAX)
                return set_err(ctx, MT_ERR_ARG, "a level box above 2^31 cells");
        }
        if (sp->coarse[0] * sp->coarse[1] * sp->coarse[2] > INT32_MAX)
            return set_err(ctx, MT_ERR_ARG, "a level box above 2^31 cells");
    }
    MT_CUDA(ctx, cudaSetDevice(ctx.device));
    rc = amr_generate(ctx, *c, *sp);
    if (rc) {
        for (int l = 0; l <= L; ++l) {
            Level &lv = c->lv[l];
            if (lv.draw_keys) cudaFreeAsync(lv.draw_keys, ctx.stream);
            if (lv.draw_set) cudaFreeAsync(lv.draw_set, ctx.stream);
            lv.draw_keys = nullptr;
            lv.draw_set = nullptr;
            lv.ndraw = 0;
        }
        if (c->dis_key) cudaFreeAsync(c->dis_key, ctx.stream);
        if (c->dis) cudaFreeAsync(c->dis, ctx.stream);
        c->dis_key = nullptr;
        c->dis = nullptr;
        c->ndis = 0;
        c->dis_on_device = false;
        return rc;
    }
    rc = amr_build(ctx, *c);
    if (rc) return rc;
    const double u0[3] = {c->d.u_bc[0], c->d.u_bc[1], c->d.u_bc[2]};
    rc = amr_init_equilibrium(ctx, *c, c->d.rho0, u0);
    if (rc) return rc;
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}

int mt_case_remap(mt_ctx *h, int32_t dst_id, int32_t src_id, int64_t *counts)
{
    Case *d, *s;
    int rc = get_case(h, dst_id, &d);
    if (rc) return rc;
    if ((rc = get_case(h, src_id, &s))) return rc;
    Ctx &ctx = h->c;
    if (d == s) return set_err(ctx, MT_ERR_ARG, "remap needs two cases");
    if (d->dense || s->dense || !d->built || !s->built) return set_err(ctx, MT_ERR_STATE, "remap needs two built multi-level cases");
    if (d->d.q != s->d.q || d->d.max_level != s->d.max_level || d->d.storage != s->d.storage)
        return set_err(ctx, MT_ERR_ARG, "remap needs the same lattice (Q), level count and storage");
    for (int a = 0; a < 3; ++a)
        if (d->d.extent0[a] != s->d.extent0[a]) return set_err(ctx, MT_ERR_ARG, "remap needs the same level-0 extent");
    if (d->in_batch || s->in_batch) return set_err(ctx, MT_ERR_STATE, "remap of a batch member");
    MT_CUDA(ctx, cudaSetDevice(ctx.device));
    return amr_remap(ctx, *d, *s, counts);
}

int mt_case_level_size(mt_ctx *h, int32_t id, int32_t level, int64_t *n)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    if (!n || level < 0 || level > c->d.max_level) return set_err(h->c, MT_ERR_ARG, "bad level");
    *n = c->dense ? c->N : c->lv[level].n;
    return MT_OK;
}

int mt_case_get_keys(mt_ctx *h, int32_t id, int32_t level, uint64_t *keys, uint32_t *tags)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense) {
        // the dense cube is every key 0 .. N-1 (level 0, Morton order), all lat_f
        for (int64_t i = 0; i < c->N; ++i) {
            if (keys) keys[i] = (uint64_t)i;
            if (tags) tags[i] = TAG_LATF;
        }
        return MT_OK;
    }
    if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
    if (level < 0 || level > c->d.max_level) return set_err(ctx, MT_ERR_ARG, "bad level");
    Level &lv = c->lv[level];
    if (lv.n == 0) return MT_OK;
    if (keys) MT_CUDA(ctx, cudaMemcpyAsync(keys, lv.key, 8 * lv.n, cudaMemcpyDeviceToHost, ctx.stream));
    if (tags) MT_CUDA(ctx, cudaMemcpyAsync(tags, lv.tag, 4 * lv.n, cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}

int mt_case_get_neighbors(mt_ctx *h, int32_t id, int32_t level, int32_t *nbr)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || !c->built) return set_err(ctx, MT_ERR_STATE, "neighbour tables exist for built multi-level cases");
    if (level < 0 || level > c->d.max_level || !nbr) return set_err(ctx, MT_ERR_ARG, "bad level");
    Level &lv = c->lv[level];
    if (lv.n == 0) return MT_OK;
    MT_CUDA(ctx, cudaMemcpyAsync(nbr, lv.nbr, 4 * lv.n * (c->d.q - 1), cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}

int mt_find(mt_ctx *h, int32_t id, int32_t level, const uint64_t *keys, int64_t n, int64_t *idx)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (n < 0 || (n > 0 && (!keys || !idx))) return set_err(ctx, MT_ERR_ARG, "bad arrays");
    if (c->dense) {
        for (int64_t i = 0; i < n; ++i) idx[i] = keys[i] < (uint64_t)c->N ? (int64_t)keys[i] : -1;
        return MT_OK;
    }
    if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
    if (level < 0 || level > c->d.max_level) return set_err(ctx, MT_ERR_ARG, "bad level");
    return amr_find(ctx, *c, level, keys, n, idx);
}

int mt_case_init_equilibrium(mt_ctx *h, int32_t id, double rho0, const double *u0)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!u0) return set_err(ctx, MT_ERR_ARG, "null velocity");
    if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
    if (c->dense)
        return dense_dispatch(*c, [&](auto *tag) {
            using S = std::remove_pointer_t<decltype(tag)>;
            return DenseOps<S>::init(ctx, *c, nullptr, nullptr, nullptr, nullptr, rho0, u0);
        });
    c->primed = false;
    c->f_stale = false;  // every f is rewritten
    return amr_init_equilibrium(ctx, *c, rho0, u0);
}

int mt_case_init_fields(mt_ctx *h, int32_t id, const double *rho, const double *ux, const double *uy,
                        const double *uz)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!c->dense) return set_err(ctx, MT_ERR_STATE, "field initialisation is for the dense path");
    if (!rho || !ux || !uy || !uz) return set_err(ctx, MT_ERR_ARG, "null field");
    double *d = nullptr;
    const size_t nb = sizeof(double) * c->N;
    MT_CUDA(ctx, cudaMallocAsync(&d, 4 * nb, ctx.stream));
    MT_CUDA(ctx, cudaMemcpyAsync(d, rho, nb, cudaMemcpyHostToDevice, ctx.stream));
    MT_CUDA(ctx, cudaMemcpyAsync(d + c->N, ux, nb, cudaMemcpyHostToDevice, ctx.stream));
    MT_CUDA(ctx, cudaMemcpyAsync(d + 2 * c->N, uy, nb, cudaMemcpyHostToDevice, ctx.stream));
    MT_CUDA(ctx, cudaMemcpyAsync(d + 3 * c->N, uz, nb, cudaMemcpyHostToDevice, ctx.stream));
    const double u0[3] = {0, 0, 0};
    rc = dense_dispatch(*c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return DenseOps<S>::init(ctx, *c, d, d + c->N, d + 2 * c->N, d + 3 * c->N, 1.0, u0);
    });
    cudaFreeAsync(d, ctx.stream);
    return rc;
}

int mt_case_set_populations(mt_ctx *h, int32_t id, int32_t level, const double *f, const double *fcol)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
    if (level < 0 || level > c->d.max_level) return set_err(ctx, MT_ERR_ARG, "bad level");
    const int Q = c->d.q;
    if (c->dense) {
        if (!f) return set_err(ctx, MT_ERR_ARG, "null populations");
        if (fcol && fcol != f && std::memcmp(f, fcol, sizeof(double) * Q * c->N) != 0)
            return set_err(ctx, MT_ERR_ARG, "the dense path starts from f == fcol");
        double *d = nullptr;
        MT_CUDA(ctx, cudaMallocAsync(&d, sizeof(double) * Q * c->N, ctx.stream));
        MT_CUDA(ctx, cudaMemcpyAsync(d, f, sizeof(double) * Q * c->N, cudaMemcpyHostToDevice, ctx.stream));
        rc = dense_dispatch(*c, [&](auto *tag) {
            using S = std::remove_pointer_t<decltype(tag)>;
            return DenseOps<S>::set(ctx, *c, d);
        });
        cudaFreeAsync(d, ctx.stream);
        return rc;
    }
    c->primed = false;
    return amr_set(ctx, *c, level, f, fcol);
}

int mt_case_get_populations(mt_ctx *h, int32_t id, int32_t level, double *f, double *fcol)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
    if (level < 0 || level > c->d.max_level) return set_err(ctx, MT_ERR_ARG, "bad level");
    const int Q = c->d.q;
    if (c->dense) {
        double *d = nullptr;
        const size_t nb = sizeof(double) * Q * c->N;
        MT_CUDA(ctx, cudaMallocAsync(&d, nb, ctx.stream));
        for (int which = 0; which < 2; ++which) {
            double *dst = which == 0 ? f : fcol;
            if (!dst) continue;
            const int pull = (which == 0 && c->a_is_fcol) ? 1 : 0;
            rc = dense_dispatch(*c, [&](auto *tag) {
                using S = std::remove_pointer_t<decltype(tag)>;
                return DenseOps<S>::get(ctx, *c, d, pull);
            });
            if (rc) break;
            MT_CUDA(ctx, cudaMemcpyAsync(dst, d, nb, cudaMemcpyDeviceToHost, ctx.stream));
        }
        MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
        cudaFreeAsync(d, ctx.stream);
        return rc;
    }
    return amr_get(ctx, *c, level, f, fcol);
}

int mt_case_get_macros(mt_ctx *h, int32_t id, int32_t level, double *rho, double *u)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
    if (level < 0 || level > c->d.max_level) return set_err(ctx, MT_ERR_ARG, "bad level");
    if (c->dense) {
        double *d = nullptr;
        MT_CUDA(ctx, cudaMallocAsync(&d, sizeof(double) * 4 * c->N, ctx.stream));
        rc = dense_dispatch(*c, [&](auto *tag) {
            using S = std::remove_pointer_t<decltype(tag)>;
            return DenseOps<S>::macros(ctx, *c, d, d + c->N);
        });
        if (!rc) {
            if (rho) MT_CUDA(ctx, cudaMemcpyAsync(rho, d, sizeof(double) * c->N, cudaMemcpyDeviceToHost, ctx.stream));
            if (u) MT_CUDA(ctx, cudaMemcpyAsync(u, d + c->N, sizeof(double) * 3 * c->N, cudaMemcpyDeviceToHost, ctx.stream));
        }
        MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
        cudaFreeAsync(d, ctx.stream);
        return rc;
    }
    return amr_macros(ctx, *c, level, rho, u);
}

int mt_case_reduce_levels(mt_ctx *h, int32_t id, double *out)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!out) return set_err(ctx, MT_ERR_ARG, "null output");
    if (c->dense) {
        // one level: its row and the total are the same sums
        rc = mt_case_reduce(h, id, out);
        if (!rc)
            for (int k = 0; k < 5; ++k) out[5 + k] = out[k];
        return rc;
    }
    if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
    return amr_reduce(ctx, *c, out);
}

int mt_case_info(mt_ctx *h, int32_t id, double *out)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!out) return set_err(ctx, MT_ERR_ARG, "null output");
    if (c->dense) return set_err(ctx, MT_ERR_STATE, "the info diagnostics belong to multi-level cases");
    if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
    return amr_info(ctx, *c, out);
}

int mt_case_reduce(mt_ctx *h, int32_t id, double *out)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!out) return set_err(ctx, MT_ERR_ARG, "null output");
    if (!c->dense) {
        // the volume-weighted total row of the per-level reduction
        if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
        std::vector<double> rows(5 * (size_t)(c->d.max_level + 2));
        rc = amr_reduce(ctx, *c, rows.data());
        if (!rc)
            for (int k = 0; k < 5; ++k) out[k] = rows[5 * (size_t)(c->d.max_level + 1) + k];
        return rc;
    }
    double *d = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&d, sizeof(double) * 5, ctx.stream));
    rc = dense_dispatch(*c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return DenseOps<S>::reduce(ctx, *c, d);
    });
    if (!rc) MT_CUDA(ctx, cudaMemcpyAsync(out, d, sizeof(double) * 5, cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    cudaFreeAsync(d, ctx.stream);
    return rc;
}

int mt_calculate_macros(mt_ctx *h, int32_t id, int32_t level) { return phase_call(h, id, PH_MACROS, level); }
int mt_collide(mt_ctx *h, int32_t id, int32_t level) { return phase_call(h, id, PH_COLLIDE, level); }
int mt_stream(mt_ctx *h, int32_t id, int32_t level) { return phase_call(h, id, PH_STREAM, level); }
int mt_explosion(mt_ctx *h, int32_t id, int32_t level) { return phase_call(h, id, PH_EXPLOSION, level); }
int mt_coalescence(mt_ctx *h, int32_t id, int32_t level) { return phase_call(h, id, PH_COALESCENCE, level); }
int mt_apply_bc(mt_ctx *h, int32_t id)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    return phase_call(h, id, c->d.bc_mode == MT_BC_NEQ ? PH_BC : (c->d.bc_mode == MT_BC_ZOUHE_HH ? PH_BC_HH : PH_BC_INOUT),
                      0);
}
int mt_apply_bc_face(mt_ctx *h, int32_t id, int32_t face)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    if (face < 0 || face > 5) return set_err(h->c, MT_ERR_ARG, "face must be 0..5 (West East South North Bot Top)");
    if (c->d.bc_mode != MT_BC_NEQ) return set_err(h->c, MT_ERR_STATE, "per-face calls apply to the NEQ boundary");
    return phase_call(h, id, PH_BC_FACE0 + face, 0);
}

int mt_ib_treat(mt_ctx *h, int32_t id)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    return phase_call(h, id, PH_IB, c->d.max_level);
}

int mt_lbm_kernel(mt_ctx *h, int32_t id, int32_t level)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || !c->built) return set_err(ctx, MT_ERR_STATE, "LBMkernel needs a built multi-level case");
    if (level < 0 || level > c->d.max_level) return set_err(ctx, MT_ERR_ARG, "bad level");
    if ((rc = amr_sync_f(ctx, *c))) return rc;
    c->primed = false;
    return amr_lbm_kernel(ctx, *c, level);
}

int mt_step(mt_ctx *h, int32_t id, int32_t n)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
    if (n < 0) return set_err(ctx, MT_ERR_ARG, "negative step count");
    if (n == 0) return MT_OK;
    if (c->dense) {
        rc = dense_dispatch(*c, [&](auto *tag) {
            using S = std::remove_pointer_t<decltype(tag)>;
            int r = MT_OK, left = n;
            if (!c->a_is_fcol) {
                r = DenseOps<S>::step(ctx, *c, 1);
                if (r) return r;
                c->a_is_fcol = true;
                --left;
            }
            for (int s = 0; s < left && !r; ++s) r = DenseOps<S>::step(ctx, *c, 0);
            return r;
        });
        if (!rc) c->coarse_steps += n;
        return rc;
    }
    if (c->in_batch) return set_err(ctx, MT_ERR_STATE, "the case belongs to a batch: step it with mt_batch_step");
    rc = amr_step(ctx, *c, n);
    if (rc) return rc;
    c->coarse_steps += n;
    return MT_OK;
}

int mt_case_get_step(mt_ctx *h, int32_t id, int64_t *coarse_steps)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    if (!coarse_steps) return set_err(h->c, MT_ERR_ARG, "null output");
    *coarse_steps = c->coarse_steps;
    return MT_OK;
}

// the direct-forcing force field of the finest level (fixed point, 2^-32)
static int df_field(mt_ctx *h, int32_t id, Case **out)
{
    int rc = get_case(h, id, out);
    if (rc) return rc;
    if (!(*out)->built) return set_err(h->c, MT_ERR_STATE, "case not built");
    if (!(*out)->acc) return set_err(h->c, MT_ERR_STATE, "not a direct-forcing case");
    return MT_OK;
}

int mt_case_get_df_force_field(mt_ctx *h, int32_t id, int64_t *out)
{
    Case *c;
    int rc = df_field(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!out) return set_err(ctx, MT_ERR_ARG, "null output");
    const size_t nb = sizeof(long long) * 3 * (size_t)c->lv[c->d.max_level].n;
    MT_CUDA(ctx, cudaMemcpyAsync(out, c->acc, nb, cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}

int mt_case_set_df_force_field(mt_ctx *h, int32_t id, const int64_t *in)
{
    Case *c;
    int rc = df_field(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!in) return set_err(ctx, MT_ERR_ARG, "null input");
    const size_t nb = sizeof(long long) * 3 * (size_t)c->lv[c->d.max_level].n;
    MT_CUDA(ctx, cudaMemcpyAsync(c->acc, in, nb, cudaMemcpyHostToDevice, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    c->primed = false;  // the band's next collision takes this force
    return MT_OK;
}

int mt_case_set_step(mt_ctx *h, int32_t id, int64_t coarse_steps)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (coarse_steps < 0) return set_err(ctx, MT_ERR_ARG, "negative step count");
    if (c->tstep) {
        // the markers' path is indexed by the finest substeps taken
        const long long t = (long long)(coarse_steps << c->d.max_level);
        MT_CUDA(ctx, cudaMemcpyAsync(c->tstep, &t, sizeof(t), cudaMemcpyHostToDevice, ctx.stream));
        MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    }
    c->coarse_steps = coarse_steps;
    return MT_OK;
}

int mt_case_set_schedule(mt_ctx *h, int32_t id, int32_t schedule)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense) return set_err(ctx, MT_ERR_STATE, "the dense path has a single (fused) schedule");
    if (schedule != MT_SCHED_PHASES && schedule != MT_SCHED_FUSED && schedule != MT_SCHED_FUSED_LISTS)
        return set_err(ctx, MT_ERR_ARG, "schedule must be MT_SCHED_PHASES, MT_SCHED_FUSED or MT_SCHED_FUSED_LISTS");
    if (schedule != MT_SCHED_PHASES && c->d.bc_mode == MT_BC_ZOUHE_HH)
        return set_err(ctx, MT_ERR_ARG, "the Zou-He / Hecht-Harting boundary runs under the phase schedule");
    const bool bricks = schedule == MT_SCHED_FUSED;
    if (!c->dense && c->built && (rc = amr_sync_f(ctx, *c))) return rc;
    if (schedule == MT_SCHED_PHASES) {
        c->primed = false;
        c->schedule = MT_SCHED_PHASES;
        return MT_OK;
    }
    if (c->schedule == MT_SCHED_PHASES || bricks != c->use_bricks) {
        c->primed = false;
        // the fused graphs bake in the pass each level uses
        amr_drop_fused(*c);
    }
    c->use_bricks = bricks;
    c->schedule = MT_SCHED_FUSED;
    return MT_OK;
}

int mt_case_set_interface_scaling(mt_ctx *h, int32_t id, int32_t scaling)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense) return set_err(ctx, MT_ERR_STATE, "the dense path has no level interface");
    if (scaling != MT_SCALE_REFERENCE && scaling != MT_SCALE_STANDARD)
        return set_err(ctx, MT_ERR_ARG, "scaling must be MT_SCALE_REFERENCE or MT_SCALE_STANDARD");
    if (scaling != c->scaling) {
        // the captured steps bake the factors in
        if (c->graph) cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
        for (int p = 0; p < 2; ++p) {
            if (c->fgraph[p]) cudaGraphExecDestroy(c->fgraph[p]);
            c->fgraph[p] = nullptr;
        }
    }
    c->scaling = scaling;
    return MT_OK;
}

int mt_case_set_interface_time(mt_ctx *h, int32_t id, int32_t mode)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense) return set_err(ctx, MT_ERR_STATE, "the dense path has no level interface");
    if (mode != MT_ITIME_REFERENCE && mode != MT_ITIME_HOLD && mode != MT_ITIME_EXTRAP)
        return set_err(ctx, MT_ERR_ARG, "mode must be MT_ITIME_REFERENCE, MT_ITIME_HOLD or MT_ITIME_EXTRAP");
    c->prev_stale = true;
    if (mode != c->itime) {
        // the captured steps bake the explosion launches in
        if (c->graph) cudaGraphExecDestroy(c->graph);
        c->graph = nullptr;
        for (int p = 0; p < 2; ++p) {
            if (c->fgraph[p]) cudaGraphExecDestroy(c->fgraph[p]);
            c->fgraph[p] = nullptr;
        }
    }
    c->itime = mode;
    return MT_OK;
}

int mt_case_set_face_velocity(mt_ctx *h, int32_t id, int32_t face, const double *u)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || !c->built) return set_err(ctx, MT_ERR_STATE, "face velocities need a built multi-level case");
    if (face < 0 || face > 5) return set_err(ctx, MT_ERR_ARG, "face must be 0..5 (West East South North Bot Top)");
    if (!u) return set_err(ctx, MT_ERR_ARG, "null velocity");
    return amr_set_face(ctx, *c, face, u);
}

int mt_case_set_markers(mt_ctx *h, int32_t id, int64_t nm, const double *ref, const double *dv, const double *center,
                        int64_t period, const double *path)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || !c->built) return set_err(ctx, MT_ERR_STATE, "markers need a built multi-level case");
    if (c->d.ib_method != MT_IB_DF) return set_err(ctx, MT_ERR_STATE, "markers need ib_method MT_IB_DF");
    if (!c->lv[c->d.max_level].nband) return set_err(ctx, MT_ERR_MESH, "no MT_SET_IB_BAND cells on the finest level");
    if (nm < 0 || period < 1 || (nm && (!ref || !dv)) || !center || !path)
        return set_err(ctx, MT_ERR_ARG, "bad marker arrays");
    void *old[] = {c->mref, c->mdv, c->path, c->mforce, c->mgrid};
    for (void *p : old)
        if (p) cudaFree(p);
    c->mref = c->mdv = c->path = c->mforce = nullptr;
    c->mgrid = nullptr;
    c->nm = nm;
    c->period = period;
    for (int a = 0; a < 3; ++a) c->center[a] = center[a];
    MT_CUDA(ctx, cudaMalloc(&c->path, sizeof(double) * 6 * period));
    MT_CUDA(ctx, cudaMemcpy(c->path, path, sizeof(double) * 6 * period, cudaMemcpyHostToDevice));
    if (nm) {
        MT_CUDA(ctx, cudaMalloc(&c->mref, sizeof(double) * 3 * nm));
        MT_CUDA(ctx, cudaMalloc(&c->mdv, sizeof(double) * nm));
        // per-marker forces [3][nm], the body-force partials of 256-marker
        // blocks [3][ceil(nm / 256)], and the finished-block counter of the sum
        const int64_t nbf = 3 * (nm + (nm + 255) / 256) + 1;
        MT_CUDA(ctx, cudaMalloc(&c->mforce, sizeof(double) * nbf));
        MT_CUDA(ctx, cudaMemset(c->mforce, 0, sizeof(double) * nbf));
        MT_CUDA(ctx, cudaMemcpy(c->mref, ref, sizeof(double) * 3 * nm, cudaMemcpyHostToDevice));
        MT_CUDA(ctx, cudaMemcpy(c->mdv, dv, sizeof(double) * nm, cudaMemcpyHostToDevice));
    }
    MT_CUDA(ctx, cudaMemsetAsync(c->tstep, 0, sizeof(long long), ctx.stream));
    if (nm) {
        // the box every marker stencil can reach over the path: centre + path
        // extent +- (largest marker offset + 2.5 cells)
        double rmax = 0.0, pmin[3] = {0, 0, 0}, pmax[3] = {0, 0, 0};
        for (int64_t m = 0; m < nm; ++m) {
            const double r2 = ref[m] * ref[m] + ref[nm + m] * ref[nm + m] + ref[2 * nm + m] * ref[2 * nm + m];
            rmax = std::max(rmax, std::sqrt(r2));
        }
        for (int64_t t = 0; t < period; ++t)
            for (int a = 0; a < 3; ++a) {
                pmin[a] = std::min(pmin[a], path[6 * t + a]);
                pmax[a] = std::max(pmax[a], path[6 * t + a]);
            }
        int64_t total = 1;
        for (int a = 0; a < 3; ++a) {
            const int64_t lo = std::max<int64_t>(0, (int64_t)std::floor(center[a] + pmin[a] - rmax - 3.0));
            const int64_t hi = (int64_t)std::ceil(center[a] + pmax[a] + rmax + 3.0);
            c->mlo[a] = lo;
            c->mdim[a] = std::max<int64_t>(1, hi - lo);
            total *= c->mdim[a];
        }
        MT_CUDA(ctx, cudaMalloc(&c->mgrid, sizeof(int32_t) * total));
        MT_CUDA(ctx, cudaMemsetAsync(c->mgrid, 0xff, sizeof(int32_t) * total, ctx.stream));
        if ((rc = amr_phase(ctx, *c, PH_BAND_GRID, c->d.max_level))) return rc;
    }
    // the captured steps bake the marker arrays in
    if (c->graph) cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
    for (int p = 0; p < 2; ++p) {
        if (c->fgraph[p]) cudaGraphExecDestroy(c->fgraph[p]);
        c->fgraph[p] = nullptr;
    }
    for (Batch *b : ctx.batches)
        if (b)
            for (int32_t x : b->ids)
                if (x == id) batch_drop(*b);
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}

int mt_case_prepare(mt_ctx *h, int32_t id)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || !c->built) return set_err(ctx, MT_ERR_STATE, "prepare needs a built multi-level case");
    if (c->d.bc_mode == MT_BC_ZOUHE_HH)
        return set_err(ctx, MT_ERR_ARG, "the Zou-He / Hecht-Harting boundary runs under the phase schedule");
    if ((rc = amr_sync_f(ctx, *c))) return rc;
    if (c->schedule != MT_SCHED_FUSED) {
        c->schedule = MT_SCHED_FUSED;
        c->primed = false;
    }
    if ((rc = amr_prime(ctx, *c))) return rc;
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}

int mt_case_transfer(mt_ctx *src, int32_t id, mt_ctx *dst, int32_t *new_id)
{
    Case *c;
    int rc = get_case(src, id, &c);
    if (rc) return rc;
    if (!dst || !new_id) return set_err(src->c, MT_ERR_ARG, "null destination");
    if (dst->c.device != src->c.device) return set_err(src->c, MT_ERR_ARG, "contexts on different devices");
    if (c->in_batch) return set_err(src->c, MT_ERR_STATE, "remove the case from its batches first");
    MT_CUDA(src->c, cudaStreamSynchronize(src->c.stream));
    src->c.cases[id] = nullptr;
    dst->c.cases.push_back(c);
    *new_id = (int32_t)dst->c.cases.size() - 1;
    return MT_OK;
}

// ---- batches ------------------------------------------------------------------
namespace {
int get_batch(mt_ctx *h, int32_t id, Batch **out)
{
    if (!h) return MT_ERR_ARG;
    if (id < 0 || id >= (int32_t)h->c.batches.size() || !h->c.batches[id])
        return set_err(h->c, MT_ERR_ARG, "no such batch");
    *out = h->c.batches[id];
    return MT_OK;
}
}  // namespace

int mt_batch_create(mt_ctx *h, int32_t *id)
{
    if (!h || !id) return MT_ERR_ARG;
    h->c.batches.push_back(new Batch());
    *id = (int32_t)h->c.batches.size() - 1;
    return MT_OK;
}

int mt_batch_destroy(mt_ctx *h, int32_t id)
{
    Batch *b;
    int rc = get_batch(h, id, &b);
    if (rc) return rc;
    for (int32_t cid : b->ids) {
        Case *c;
        if (!get_case(h, cid, &c)) c->in_batch--;
    }
    cudaStreamSynchronize(h->c.stream);
    batch_free(*b);
    delete b;
    h->c.batches[id] = nullptr;
    return MT_OK;
}

int mt_batch_add(mt_ctx *h, int32_t id, int32_t case_id)
{
    Batch *b;
    int rc = get_batch(h, id, &b);
    if (rc) return rc;
    Case *c;
    if ((rc = get_case(h, case_id, &c))) return rc;
    Ctx &ctx = h->c;
    if (c->dense || !c->built) return set_err(ctx, MT_ERR_STATE, "batches hold built multi-level cases");
    if (c->d.bc_mode == MT_BC_ZOUHE_HH)
        return set_err(ctx, MT_ERR_ARG, "the Zou-He / Hecht-Harting boundary runs under the phase schedule");
    for (int32_t x : b->ids)
        if (x == case_id) return set_err(ctx, MT_ERR_ARG, "the case is already in the batch");
    if ((rc = amr_sync_f(ctx, *c))) return rc;
    if (c->schedule != MT_SCHED_FUSED) {
        c->schedule = MT_SCHED_FUSED;
        c->primed = false;
    }
    if ((rc = amr_prime(ctx, *c))) return rc;
    b->ids.push_back(case_id);
    c->in_batch++;
    batch_drop(*b);
    return MT_OK;
}

int mt_batch_remove(mt_ctx *h, int32_t id, int32_t case_id)
{
    Batch *b;
    int rc = get_batch(h, id, &b);
    if (rc) return rc;
    for (size_t k = 0; k < b->ids.size(); ++k)
        if (b->ids[k] == case_id) {
            b->ids.erase(b->ids.begin() + k);
            Case *c;
            if (!get_case(h, case_id, &c)) c->in_batch--;
            batch_drop(*b);
            return MT_OK;
        }
    return set_err(h->c, MT_ERR_ARG, "the case is not in the batch");
}

int mt_batch_size(mt_ctx *h, int32_t id, int32_t *n)
{
    Batch *b;
    int rc = get_batch(h, id, &b);
    if (rc) return rc;
    if (!n) return set_err(h->c, MT_ERR_ARG, "null output");
    *n = (int32_t)b->ids.size();
    return MT_OK;
}

int mt_batch_step(mt_ctx *h, int32_t id, int32_t n)
{
    Batch *b;
    int rc = get_batch(h, id, &b);
    if (rc) return rc;
    if (n < 0) return set_err(h->c, MT_ERR_ARG, "negative step count");
    std::vector<Case *> cs;
    for (int32_t cid : b->ids) {
        Case *c;
        if ((rc = get_case(h, cid, &c))) return rc;
        cs.push_back(c);
    }
    rc = batch_step(h->c, *b, cs, n);
    if (!rc)
        for (Case *c : cs) c->coarse_steps += n;
    return rc;
}

int mt_case_status(mt_ctx *h, int32_t id)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!c->built) return set_err(ctx, MT_ERR_STATE, "case not built");
    if (c->dense) {
        double r[5];
        rc = mt_case_reduce(h, id, r);
        if (rc) return rc;
        for (double v : r)
            if (!std::isfinite(v)) return set_err(ctx, MT_ERR_NONFINITE, "non-finite population in the dense state");
        return MT_OK;
    }
    int flags = 0;
    rc = amr_guard(ctx, *c, &flags);
    if (rc) return rc;
    if (flags & DEVERR_NONFINITE) return set_err(ctx, MT_ERR_NONFINITE, "non-finite population found by the guard");
    if (flags & DEVERR_MISSING_BC_NBR)
        return set_err(ctx, MT_ERR_MESH, "a boundary cell's reserved neighbour is not stored");
    return MT_OK;
}

int mt_case_tune(mt_ctx *h, int32_t id, int32_t *best_block, float *ms_per_candidate)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!c->dense) return set_err(ctx, MT_ERR_STATE, "the tuner picks the block shape of the dense kernel");
    float ms[8];
    int blocks[8], n = 0;
    rc = dense_dispatch(*c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return DenseOps<S>::tune(ctx, *c, ms, blocks, &n);
    });
    if (rc) return rc;
    if (best_block) *best_block = c->dense_block;
    if (ms_per_candidate)
        for (int j = 0; j < n; ++j) ms_per_candidate[j] = ms[j];
    return MT_OK;
}

int mt_case_tune_bricks(mt_ctx *h, int32_t id, int32_t *variant, float *ms)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || !c->built) return set_err(ctx, MT_ERR_STATE, "the brick tuner needs a built multi-level case");
    if (c->d.bc_mode == MT_BC_ZOUHE_HH)
        return set_err(ctx, MT_ERR_ARG, "the Zou-He / Hecht-Harting boundary runs under the phase schedule");
    const int prev = c->schedule;
    if (c->schedule != MT_SCHED_FUSED) {
        // the brick tables are built with the fused schedule
        if ((rc = mt_case_set_schedule(h, id, MT_SCHED_FUSED))) return rc;
    }
    if ((rc = amr_prime(ctx, *c))) return rc;
    rc = amr_dispatch(*c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return AmrOps<S>::tune_bricks(ctx, *c, variant, ms);
    });
    if (rc) return rc;
    // the captured steps bake the kernel choice in
    for (int p = 0; p < 2; ++p) {
        if (c->fgraph[p]) cudaGraphExecDestroy(c->fgraph[p]);
        c->fgraph[p] = nullptr;
    }
    if (prev != MT_SCHED_FUSED) return mt_case_set_schedule(h, id, prev);
    return MT_OK;
}

int mt_case_set_brick_forms(mt_ctx *h, int32_t id, const int32_t *form)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense) return set_err(ctx, MT_ERR_STATE, "brick forms belong to multi-level cases");
    if (!form) return set_err(ctx, MT_ERR_ARG, "form is NULL");
    const bool f64 = c->d.storage == MT_STORE_F64;
    for (int l = 0; l <= c->d.max_level; ++l) {
        const int v = form[l];
        if (v >= MT_BRICK_FORMS || (v >= 0 && f64 && v != 0 && v != 3))
            return set_err(ctx, MT_ERR_ARG, "brick form " + std::to_string(v) + " is not available for this storage");
    }
    for (int l = 0; l <= c->d.max_level; ++l)
        if (form[l] >= 0) c->lv[l].brick_variant = form[l];
    // the captured steps bake the kernel choice in
    for (int p = 0; p < 2; ++p) {
        if (c->fgraph[p]) cudaGraphExecDestroy(c->fgraph[p]);
        c->fgraph[p] = nullptr;
    }
    return MT_OK;
}

int mt_get_force(mt_ctx *h, int32_t id, double *out4)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!out4) return set_err(ctx, MT_ERR_ARG, "null output");
    if (c->dense || !c->force_acc) {
        for (int i = 0; i < 4; ++i) out4[i] = 0;
        return MT_OK;
    }
    MT_CUDA(ctx, cudaMemcpyAsync(out4, c->force_acc, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}

int mt_case_force_async(mt_ctx *h, int32_t id)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->dense || !c->force_acc) return set_err(ctx, MT_ERR_STATE, "the case has no force accumulator");
    if (!c->h_force) {
        MT_CUDA(ctx, cudaHostAlloc((void **)&c->h_force, 6 * sizeof(double), cudaHostAllocDefault));
        for (int i = 0; i < 6; ++i) c->h_force[i] = 0.0;
    }
    MT_CUDA(ctx, cudaMemcpyAsync(c->h_force, c->force_acc, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    // the state's guard, stream-ordered behind the same steps: flags land
    // beside the force copy
    MT_CUDA(ctx, cudaMemsetAsync(c->dev_err, 0, sizeof(int), ctx.stream));
    rc = amr_dispatch(*c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return AmrOps<S>::guard(ctx, *c, true);
    });
    if (rc) return rc;
    MT_CUDA(ctx, cudaMemcpyAsync((int *)(c->h_force + 4), c->dev_err, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    return MT_OK;
}

int mt_case_status_copied(mt_ctx *h, int32_t id)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!c->h_force) return set_err(ctx, MT_ERR_STATE, "no status copy was requested (mt_case_force_async)");
    const int flags = *(const int *)(c->h_force + 4);
    if (flags & DEVERR_NONFINITE) return set_err(ctx, MT_ERR_NONFINITE, "non-finite population found by the guard");
    return MT_OK;
}

int mt_case_force_copied(mt_ctx *h, int32_t id, double *out4)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!out4) return set_err(ctx, MT_ERR_ARG, "null output");
    if (!c->h_force) return set_err(ctx, MT_ERR_STATE, "no force copy was requested (mt_case_force_async)");
    for (int i = 0; i < 4; ++i) out4[i] = c->h_force[i];
    return MT_OK;
}

int mt_reset_force(mt_ctx *h, int32_t id)
{
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (c->force_acc) MT_CUDA(ctx, cudaMemsetAsync(c->force_acc, 0, 4 * sizeof(double), ctx.stream));
    return MT_OK;
}

}  // extern "C"

// ---- allocation-free reduction ------------------------------------------
//
// mt_case_reduce_noalloc is for callers that must not allocate device memory
// while they run: a host that has carved the GPU's memory up front for its
// cases (an admission budget, a pool shared with other processes) or that
// calls in from a context where cudaMalloc / cudaMallocAsync would take a
// driver lock or grow a pool at a bad moment.  It launches the same two
// kernels as mt_case_reduce, with their scratch in the static device array
// below instead of a cudaMallocAsync'd buffer.
//
// Scratch: 5 * MT_NOALLOC_REDUCE_BLOCKS per-block partial sums (one block per
// 256 cells) followed by the 5 totals, 640 KiB + 64 B in all; cases of more
// than 256 * MT_NOALLOC_REDUCE_BLOCKS = 4,194,304 cells are rejected with
// MT_ERR_ARG.  Nothing in it has to start at zero: each call writes every
// partial slot it reads (k_dense_reduce, blocks 0 .. ceil(N/256)-1) and then
// the 5 totals (k_sum_partials) before copying them out, in stream order.
// The array is one per device and process, so calls that overlap in time on
// the same device (two host threads, or two contexts on different streams)
// race on it; the caller serialises them.  The first call on a device looks
// up the array's device address (cudaGetSymbolAddress, with that device
// current) and caches it; make that first call before any stream capture.

namespace {

constexpr int64_t MT_NOALLOC_REDUCE_BLOCKS = 16384;
constexpr int MT_NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_reduce_scratch[5 * MT_NOALLOC_REDUCE_BLOCKS + 8];

std::mutex g_scratch_mu;
double *g_scratch_ptr[MT_NOALLOC_MAX_DEVICES] = {};

// device address of g_reduce_scratch on ctx.device (set-up on first use)
int noalloc_scratch(mt::Ctx &ctx, double **out)
{
    if (ctx.device < 0 || ctx.device >= MT_NOALLOC_MAX_DEVICES)
        return mt::set_err(ctx, MT_ERR_ARG, "device index out of range for the static reduction scratch");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[ctx.device]) {
        // the lookup needs ctx.device current; the caller's current device is
        // put back afterwards, so the set-up leaves no trace on the thread
        int prev = -1;
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) return mt::set_err(ctx, MT_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        e = cudaSetDevice(ctx.device);
        if (e != cudaSuccess) return mt::set_err(ctx, MT_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
        double *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_reduce_scratch);
        cudaError_t r = cudaSetDevice(prev);
        if (e != cudaSuccess || !p)
            return mt::set_err(ctx, MT_ERR_CUDA,
                               std::string("cudaGetSymbolAddress(reduction scratch): ") + cudaGetErrorString(e));
        if (r != cudaSuccess)
            return mt::set_err(ctx, MT_ERR_CUDA, std::string("cudaSetDevice (restore): ") + cudaGetErrorString(r));
        g_scratch_ptr[ctx.device] = p;
    }
    *out = g_scratch_ptr[ctx.device];
    return MT_OK;
}

}  // namespace

extern "C" int mt_case_reduce_noalloc(mt_ctx *h, int32_t id, double *out)
{
    using namespace mt;
    Case *c;
    int rc = get_case(h, id, &c);
    if (rc) return rc;
    Ctx &ctx = h->c;
    if (!out) return set_err(ctx, MT_ERR_ARG, "null output");
    if (!c->dense) return set_err(ctx, MT_ERR_STATE, "device reductions are implemented for the dense path");
    const int64_t blocks = (c->N + 255) / 256;
    if (blocks > MT_NOALLOC_REDUCE_BLOCKS)
        return set_err(ctx, MT_ERR_ARG,
                       "mt_case_reduce_noalloc: " + std::to_string(c->N) + " cells exceed the static scratch (at most " +
                           std::to_string(256 * MT_NOALLOC_REDUCE_BLOCKS) + " cells); use mt_case_reduce");
    double *scratch = nullptr;
    rc = noalloc_scratch(ctx, &scratch);
    if (rc) return rc;
    double *totals = scratch + 5 * MT_NOALLOC_REDUCE_BLOCKS;
    rc = dense_dispatch(*c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return DenseOps<S>::reduce_into(ctx, *c, scratch, totals);
    });
    if (rc) return rc;
    MT_CUDA(ctx, cudaMemcpyAsync(out, totals, sizeof(double) * 5, cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}
