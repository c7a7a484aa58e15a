// Multi-level path: device build of the Morton-sorted SoA levels and the
// per-phase FP64 kernels of the reference time step.
//
// Compiled with --fmad=false: every FP64 expression keeps the reference's
// operation order and rounding, so results match its CPU path bit-for-bit.
//
// Layout per level: cells sorted by Morton key; populations f/fcol as
// [Q][n] doubles; nbr as [(Q-1)][n] int32 (index of key + e_k or -1);
// index lists (int32) for each reference set in ascending key order.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "mt_internal.hpp"

namespace mt {

// ----------------------------------------------------------------------------
// build kernels
// ----------------------------------------------------------------------------
__global__ void k_tag_cells(const uint64_t *raw, const uint8_t *set, int64_t nraw, const uint64_t *key, int64_t n,
                            uint32_t *tag, int8_t *bcidx)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nraw) return;
    int64_t i = find_key(key, n, raw[j]);
    if (i < 0) return;
    const uint8_t s = set[j];
    uint32_t bit;
    if (s >= 16) {
        bit = TAG_BC;
        bcidx[i] = (int8_t)(s - 16);
    } else {
        const uint32_t bits[kNumSets] = {TAG_LATF, TAG_F2C, TAG_C2F, TAG_GC2F, TAG_GF2C, TAG_SF};
        bit = bits[s];
    }
    atomicOr(&tag[i], bit);
}

template <int Q>
__global__ void k_neighbors(MortonGeom g, int level, const uint64_t *key, int64_t n, int32_t *nbr)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t k0 = key[i];
#pragma unroll
    for (int k = 1; k < Q; ++k) {
        const uint64_t nk = find_neighbor(g, k0, level, ex(k), ey(k), ez(k));
        nbr[(int64_t)(k - 1) * n + i] = (int32_t)find_key(key, n, nk);
    }
}

__global__ void k_dis_rows(const uint64_t *key, int64_t n, const uint64_t *dkey, int64_t nd, int32_t *disrow,
                           uint32_t *tag)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t r = find_key(dkey, nd, key[i]);
    disrow[i] = (int32_t)r;
    if (r >= 0) tag[i] |= TAG_IB;
}

__global__ void k_dis_check(const uint64_t *dkey, int64_t nd, const uint64_t *key, int64_t n, int *err)
{
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= nd) return;
    if (find_key(key, n, dkey[r]) < 0) atomicOr(err, DEVERR_DIS_NOT_FINEST);
}

// children of a coarse cell on the fine level, in the order of
// LBM_Manager.cpp:1074-1082: (0,0,0) (1,0,0) (0,1,0) (1,1,0) (0,0,1) (1,0,1) (0,1,1) (1,1,1)
MT_HD void children(const MortonGeom &g, uint64_t code, int fine, uint64_t *ch)
{
    const uint64_t x1 = find_neighbor(g, code, fine, 1, 0, 0);
    const uint64_t y1 = find_neighbor(g, code, fine, 0, 1, 0);
    const uint64_t xy1 = find_neighbor(g, x1, fine, 0, 1, 0);
    ch[0] = code;
    ch[1] = x1;
    ch[2] = y1;
    ch[3] = xy1;
    ch[4] = find_neighbor(g, code, fine, 0, 0, 1);
    ch[5] = find_neighbor(g, x1, fine, 0, 0, 1);
    ch[6] = find_neighbor(g, y1, fine, 0, 0, 1);
    ch[7] = find_neighbor(g, xy1, fine, 0, 0, 1);
}

// explosion children (AMR_transDDF_explosion, LBM_Manager.cpp:1072-1128):
// F2C sources need every child stored and skip children listed in dis;
// ghost sources write only children in ghost_overlap_C2F and not in dis.
__global__ void k_expl_children(MortonGeom g, int fine, const int32_t *src, int64_t nsrc, int64_t nf2c,
                                const uint64_t *ckey, const uint64_t *fkey, const uint32_t *ftag, int64_t nf,
                                const uint64_t *dkey, int64_t nd, int32_t *child, int *err)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nsrc) return;
    uint64_t ch[8];
    children(g, ckey[src[j]], fine, ch);
    for (int m = 0; m < 8; ++m) {
        int32_t out = -1;
        const bool in_dis = find_key(dkey, nd, ch[m]) >= 0;
        const int64_t fi = find_key(fkey, nf, ch[m]);
        if (!in_dis) {
            if (j < nf2c) {
                if (fi < 0)
                    atomicOr(err, DEVERR_MISSING_CHILD);
                else
                    out = (int32_t)fi;
            } else if (fi >= 0 && (ftag[fi] & TAG_GC2F)) {
                out = (int32_t)fi;
            }
        }
        child[(int64_t)m * nsrc + j] = out;
    }
}

__global__ void k_coal_children(MortonGeom g, int fine, const int32_t *src, int64_t nsrc, const uint64_t *ckey,
                                const uint64_t *fkey, int64_t nf, int32_t *child, int *err)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nsrc) return;
    uint64_t ch[8];
    children(g, ckey[src[j]], fine, ch);
    for (int m = 0; m < 8; ++m) {
        const int64_t fi = find_key(fkey, nf, ch[m]);
        if (fi < 0) atomicOr(err, DEVERR_MISSING_CHILD);
        child[(int64_t)m * nsrc + j] = (int32_t)fi;
    }
}

struct TagHas {
    const uint32_t *tag;
    uint32_t bit;
    __host__ __device__ bool operator()(const int32_t &i) const { return (tag[i] & bit) != 0; }
};
struct BcIs {
    const int8_t *bc;
    int8_t b;
    __host__ __device__ bool operator()(const int32_t &i) const { return bc[i] == b; }
};
struct IbLatf {
    const uint32_t *tag;
    __host__ __device__ bool operator()(const int32_t &i) const
    {
        return (tag[i] & TAG_LATF) && (tag[i] & TAG_IB);
    }
};

template <class Pred>
static int select_indices(Ctx &ctx, int64_t n, Pred pred, int32_t **out, int64_t *nout)
{
    *out = nullptr;
    *nout = 0;
    if (n == 0) return MT_OK;
    int32_t *buf = nullptr;
    int *d_num = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&buf, sizeof(int32_t) * n, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&d_num, sizeof(int), ctx.stream));
    cub::CountingInputIterator<int32_t> it(0);
    size_t tmp = 0;
    MT_CUDA(ctx, cub::DeviceSelect::If(nullptr, tmp, it, buf, d_num, (int)n, pred, ctx.stream));
    void *dtmp = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&dtmp, tmp, ctx.stream));
    MT_CUDA(ctx, cub::DeviceSelect::If(dtmp, tmp, it, buf, d_num, (int)n, pred, ctx.stream));
    int h_num = 0;
    MT_CUDA(ctx, cudaMemcpyAsync(&h_num, d_num, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    cudaFreeAsync(dtmp, ctx.stream);
    cudaFreeAsync(d_num, ctx.stream);
    if (h_num == 0) {
        cudaFreeAsync(buf, ctx.stream);
        return MT_OK;
    }
    *out = buf;
    *nout = h_num;
    return MT_OK;
}

static int concat_lists(Ctx &ctx, const int32_t *a, int64_t na, const int32_t *b, int64_t nb, int32_t **out,
                        int64_t *nout)
{
    *nout = na + nb;
    *out = nullptr;
    if (*nout == 0) return MT_OK;
    MT_CUDA(ctx, cudaMallocAsync(out, sizeof(int32_t) * (*nout), ctx.stream));
    if (na) MT_CUDA(ctx, cudaMemcpyAsync(*out, a, sizeof(int32_t) * na, cudaMemcpyDeviceToDevice, ctx.stream));
    if (nb) MT_CUDA(ctx, cudaMemcpyAsync(*out + na, b, sizeof(int32_t) * nb, cudaMemcpyDeviceToDevice, ctx.stream));
    return MT_OK;
}

static int build_level(Ctx &ctx, Case &c, int l)
{
    Level &lv = c.lv[l];
    const int Q = c.d.q;
    const int64_t nraw = (int64_t)lv.raw_keys.size();
    lv.n = 0;
    if (nraw > 0) {
        uint64_t *d_raw = nullptr, *d_sorted = nullptr;
        uint8_t *d_set = nullptr;
        int *d_num = nullptr;
        MT_CUDA(ctx, cudaMallocAsync(&d_raw, 8 * nraw, ctx.stream));
        MT_CUDA(ctx, cudaMallocAsync(&d_sorted, 8 * nraw, ctx.stream));
        MT_CUDA(ctx, cudaMallocAsync(&d_set, nraw, ctx.stream));
        MT_CUDA(ctx, cudaMallocAsync(&d_num, sizeof(int), ctx.stream));
        MT_CUDA(ctx, cudaMemcpyAsync(d_raw, lv.raw_keys.data(), 8 * nraw, cudaMemcpyHostToDevice, ctx.stream));
        MT_CUDA(ctx, cudaMemcpyAsync(d_set, lv.raw_set.data(), nraw, cudaMemcpyHostToDevice, ctx.stream));
        size_t t1 = 0, t2 = 0;
        MT_CUDA(ctx, cub::DeviceRadixSort::SortKeys(nullptr, t1, d_raw, d_sorted, (int)nraw, 0, 64, ctx.stream));
        MT_CUDA(ctx, cudaMallocAsync(&lv.key, 8 * nraw, ctx.stream));
        MT_CUDA(ctx, cub::DeviceSelect::Unique(nullptr, t2, d_sorted, lv.key, d_num, (int)nraw, ctx.stream));
        void *tmp = nullptr;
        MT_CUDA(ctx, cudaMallocAsync(&tmp, std::max(t1, t2), ctx.stream));
        MT_CUDA(ctx, cub::DeviceRadixSort::SortKeys(tmp, t1, d_raw, d_sorted, (int)nraw, 0, 64, ctx.stream));
        MT_CUDA(ctx, cub::DeviceSelect::Unique(tmp, t2, d_sorted, lv.key, d_num, (int)nraw, ctx.stream));
        int h_num = 0;
        MT_CUDA(ctx, cudaMemcpyAsync(&h_num, d_num, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
        MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
        lv.n = h_num;
        const int64_t n = lv.n;
        MT_CUDA(ctx, cudaMallocAsync(&lv.tag, 4 * n, ctx.stream));
        MT_CUDA(ctx, cudaMemsetAsync(lv.tag, 0, 4 * n, ctx.stream));
        MT_CUDA(ctx, cudaMallocAsync(&lv.bcidx, n, ctx.stream));
        MT_CUDA(ctx, cudaMemsetAsync(lv.bcidx, 0xff, n, ctx.stream));
        k_tag_cells<<<grid_for(nraw, 256), 256, 0, ctx.stream>>>(d_raw, d_set, nraw, lv.key, n, lv.tag, lv.bcidx);
        MT_LAUNCHED(ctx);
        cudaFreeAsync(tmp, ctx.stream);
        cudaFreeAsync(d_raw, ctx.stream);
        cudaFreeAsync(d_sorted, ctx.stream);
        cudaFreeAsync(d_set, ctx.stream);
        cudaFreeAsync(d_num, ctx.stream);
    }
    const int64_t n = lv.n;
    if (n == 0) return MT_OK;
    MT_CUDA(ctx, cudaMallocAsync(&lv.disrow, 4 * n, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.disrow, 0xff, 4 * n, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&lv.nbr, 4 * n * (Q - 1), ctx.stream));
    if (Q == 19)
        k_neighbors<19><<<grid_for(n, 128), 128, 0, ctx.stream>>>(c.geom, l, lv.key, n, lv.nbr);
    else
        k_neighbors<27><<<grid_for(n, 128), 128, 0, ctx.stream>>>(c.geom, l, lv.key, n, lv.nbr);
    MT_LAUNCHED(ctx);
    MT_CUDA(ctx, cudaMallocAsync(&lv.f, 8 * n * Q, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&lv.fcol, 8 * n * Q, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&lv.rho, 8 * n, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&lv.u, 8 * 3 * n, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.f, 0, 8 * n * Q, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.fcol, 0, 8 * n * Q, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.rho, 0, 8 * n, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.u, 0, 8 * 3 * n, ctx.stream));
    const uint32_t bits[kNumSets] = {TAG_LATF, TAG_F2C, TAG_C2F, TAG_GC2F, TAG_GF2C, TAG_SF};
    for (int s = 0; s < kNumSets; ++s) {
        int rc = select_indices(ctx, n, TagHas{lv.tag, bits[s]}, &lv.list[s], &lv.nlist[s]);
        if (rc) return rc;
    }
    if (l == 0)
        for (int b = 0; b < 26; ++b) {
            int rc = select_indices(ctx, n, BcIs{lv.bcidx, (int8_t)b}, &lv.bclist[b], &lv.nbc[b]);
            if (rc) return rc;
        }
    int rc = concat_lists(ctx, lv.list[0], lv.nlist[0], lv.list[1], lv.nlist[1], &lv.collide_list, &lv.ncollide);
    if (rc) return rc;
    return concat_lists(ctx, lv.list[0], lv.nlist[0], lv.list[2], lv.nlist[2], &lv.stream_list, &lv.nstream);
}

int amr_build(Ctx &ctx, Case &c)
{
    const int L = c.d.max_level;
    c.geom.L = L;
    for (int a = 0; a < 3; ++a) {
        c.geom.periodic[a] = c.d.periodic[a];
        c.geom.extent0[a] = c.d.extent0[a];
    }
    MT_CUDA(ctx, cudaMallocAsync(&c.dev_err, sizeof(int), ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(c.dev_err, 0, sizeof(int), ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&c.force_acc, 4 * sizeof(double), ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(c.force_acc, 0, 4 * sizeof(double), ctx.stream));
    for (int l = 0; l <= L; ++l) {
        int rc = build_level(ctx, c, l);
        if (rc) return rc;
    }
    // dis rows and the IB cell list on the finest level
    c.ndis = (int64_t)c.h_dis_key.size();
    const int W = c.d.q - 1;
    if (c.ndis > 0) {
        MT_CUDA(ctx, cudaMallocAsync(&c.dis_key, 8 * c.ndis, ctx.stream));
        MT_CUDA(ctx, cudaMallocAsync(&c.dis, 8 * c.ndis * W, ctx.stream));
        MT_CUDA(ctx, cudaMemcpyAsync(c.dis_key, c.h_dis_key.data(), 8 * c.ndis, cudaMemcpyHostToDevice, ctx.stream));
        MT_CUDA(ctx, cudaMemcpyAsync(c.dis, c.h_dis.data(), 8 * c.ndis * W, cudaMemcpyHostToDevice, ctx.stream));
        Level &fl = c.lv[L];
        if (fl.n > 0) {
            k_dis_rows<<<grid_for(fl.n, 256), 256, 0, ctx.stream>>>(fl.key, fl.n, c.dis_key, c.ndis, fl.disrow, fl.tag);
            MT_LAUNCHED(ctx);
        }
        k_dis_check<<<grid_for(c.ndis, 256), 256, 0, ctx.stream>>>(c.dis_key, c.ndis, fl.key, fl.n, c.dev_err);
        MT_LAUNCHED(ctx);
        int rc = select_indices(ctx, fl.n, IbLatf{fl.tag}, &fl.iblist, &fl.nib);
        if (rc) return rc;
        if (fl.nib) MT_CUDA(ctx, cudaMallocAsync(&c.ib_force, 8 * 3 * fl.nib, ctx.stream));
    }
    {
        int64_t maxn = 0;
        for (int b = 0; b < 26; ++b) maxn = std::max(maxn, c.lv[0].nbc[b]);
        if (maxn) MT_CUDA(ctx, cudaMallocAsync(&c.bc_tmp, sizeof(double) * 18 * maxn, ctx.stream));
    }
    // cross-level child tables
    for (int l = 1; l <= L; ++l) {
        Level &cl = c.lv[l - 1], &fl = c.lv[l];
        int rc = concat_lists(ctx, cl.list[1], cl.nlist[1], cl.list[4], cl.nlist[4], &fl.expl_src, &fl.nexpl);
        if (rc) return rc;
        fl.nexpl_f2c = cl.nlist[1];
        if (fl.nexpl) {
            MT_CUDA(ctx, cudaMallocAsync(&fl.expl_child, 4 * 8 * fl.nexpl, ctx.stream));
            k_expl_children<<<grid_for(fl.nexpl, 128), 128, 0, ctx.stream>>>(
                c.geom, l, fl.expl_src, fl.nexpl, fl.nexpl_f2c, cl.key, fl.key, fl.tag, fl.n, c.dis_key, c.ndis,
                fl.expl_child, c.dev_err);
            MT_LAUNCHED(ctx);
        }
        if (cl.nlist[1]) {
            MT_CUDA(ctx, cudaMallocAsync(&cl.coal_child, 4 * 8 * cl.nlist[1], ctx.stream));
            k_coal_children<<<grid_for(cl.nlist[1], 128), 128, 0, ctx.stream>>>(
                c.geom, l, cl.list[1], cl.nlist[1], cl.key, fl.key, fl.n, cl.coal_child, c.dev_err);
            MT_LAUNCHED(ctx);
        }
    }
    int herr = 0;
    MT_CUDA(ctx, cudaMemcpyAsync(&herr, c.dev_err, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    if (herr & DEVERR_MISSING_CHILD)
        return set_err(ctx, MT_ERR_MESH, "a child of an overlap_F2C cell is not stored on the finer level");
    if (herr & DEVERR_DIS_NOT_FINEST) return set_err(ctx, MT_ERR_MESH, "a dis key is not a finest-level cell");
    for (int l = 0; l <= L; ++l) {
        c.lv[l].raw_keys.clear();
        c.lv[l].raw_keys.shrink_to_fit();
        c.lv[l].raw_set.clear();
        c.lv[l].raw_set.shrink_to_fit();
    }
    c.built = true;
    return MT_OK;
}

void amr_free(Case &c)
{
    for (int l = 0; l < kMaxLevels; ++l) {
        Level &lv = c.lv[l];
        void *ptrs[] = {lv.key, lv.tag, lv.bcidx, lv.disrow, lv.nbr, lv.f, lv.fcol, lv.rho, lv.u,
                        lv.collide_list, lv.stream_list, lv.iblist, lv.expl_src, lv.expl_child, lv.coal_child};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        for (int s = 0; s < kNumSets; ++s)
            if (lv.list[s]) cudaFree(lv.list[s]);
        for (int b = 0; b < 26; ++b)
            if (lv.bclist[b]) cudaFree(lv.bclist[b]);
        lv = Level();
    }
    void *ptrs[] = {c.dis_key, c.dis, c.ib_force, c.force_acc, c.dev_err, c.bc_tmp};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    c.bc_tmp = nullptr;
    c.dis_key = nullptr;
    c.dis = nullptr;
    c.ib_force = nullptr;
    c.force_acc = nullptr;
    c.dev_err = nullptr;
    if (c.graph) cudaGraphExecDestroy(c.graph);
    c.graph = nullptr;
}

// ----------------------------------------------------------------------------
// FP64 phase kernels (reference operation order)
// ----------------------------------------------------------------------------
template <int Q>
__global__ void k_init_eq(int64_t n, const uint32_t *tag, double rho0, double ux, double uy, double uz, double *f,
                          double *fcol, double *rho, double *u)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = tag[i];
    const bool solid = (t & TAG_SF) && !(t & (TAG_LATF | TAG_F2C | TAG_C2F | TAG_GC2F | TAG_BC));
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double v = solid ? 0. : feq_ref<Q>(k, rho0, ux, uy, uz);
        f[k * n + i] = v;
        fcol[k * n + i] = v;
    }
    rho[i] = solid ? 1. : rho0;
    u[i] = solid ? 0. : ux;
    u[n + i] = solid ? 0. : uy;
    u[2 * n + i] = solid ? 0. : uz;
}

// LBM_Manager::calculateMacros(level), LBM_Manager.cpp:1003-1050
template <int Q>
__global__ void k_macros(const int32_t *list, int64_t nl, int64_t n, const double *f, double *rho, double *u)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    double d[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) d[k] = f[k * n + i];
    double r, x, y, z;
    macros_ref<Q>(d, r, x, y, z);
    rho[i] = r;
    u[i] = x;
    u[n + i] = y;
    u[2 * n + i] = z;
}

// Collision_LBGK::collide / Collision_Cumulant::collide on lat_f + F2C
template <int Q, int COLL>
__global__ void k_collide(const int32_t *list, int64_t nl, int64_t n, double tau, const double *f, const double *rho,
                          const double *u, double *fcol)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    const double r = rho[i], x = u[i], y = u[n + i], z = u[2 * n + i];
    if (COLL == MT_COLL_LBGK) {
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            const double fk = f[k * n + i];
            fcol[k * n + i] = fk - (fk - feq_ref<Q>(k, r, x, y, z)) / tau;
        }
    } else {
        double d[27], o[27];
#pragma unroll
        for (int k = 0; k < 27; ++k) d[k] = f[k * n + i];
        cumulant_collide<double>(d, r, x, y, z, 1. / tau, o);
#pragma unroll
        for (int k = 0; k < 27; ++k) fcol[k * n + i] = o[k];
    }
}

// fcol = f on overlap_C2F (Collision_Manager.cpp:45-52)
template <int Q>
__global__ void k_copy_fcol(const int32_t *list, int64_t nl, int64_t n, const double *f, double *fcol)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
#pragma unroll
    for (int k = 0; k < Q; ++k) fcol[k * n + i] = f[k * n + i];
}

// ABPatternPull::stream (Stream_Manager.cpp:43-76): missing neighbour keeps f
template <int Q>
__global__ void k_stream(const int32_t *list, int64_t nl, int64_t n, int textbook, const int32_t *nbr,
                         const double *fcol, double *f)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    f[i] = fcol[i];
#pragma unroll
    for (int k = 1; k < Q; ++k) {
        const int kk = textbook ? inv(k) : k;
        const int32_t s = nbr[(int64_t)(kk - 1) * n + i];
        if (s >= 0) f[k * n + i] = fcol[k * n + s];
    }
}

// AMR_transDDF_explosion (LBM_Manager.cpp:1059-1129)
template <int Q>
__global__ void k_explosion(const int32_t *src, const int32_t *child, int64_t ns, int64_t nc, const double *cfcol,
                            int64_t nf, double *ffcol, double scale)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= ns) return;
    const int64_t i = src[j];
    double d[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) d[k] = cfcol[k * nc + i];
    double r, x, y, z;
    macros_ref<Q>(d, r, x, y, z);
    int32_t ch[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) ch[m] = child[(int64_t)m * ns + j];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double fe = feq_heluo_ref<Q>(k, r, x, y, z);
        const double v = fe + scale * (d[k] - fe);
#pragma unroll
        for (int m = 0; m < 8; ++m)
            if (ch[m] >= 0) ffcol[k * nf + ch[m]] = v;
    }
}

// AMR_transDDF_coalescence (LBM_Manager.cpp:1131-1169)
template <int Q>
__global__ void k_coalescence(const int32_t *list, const int32_t *child, int64_t nl, int64_t nc, double *cf,
                              const double *ff, int64_t nf, double scale)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    int32_t ch[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) ch[m] = child[(int64_t)m * nl + j];
    double a[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        double s = 0;
#pragma unroll
        for (int m = 0; m < 8; ++m) s += ff[k * nf + ch[m]];
        a[k] = s / 8.0;
    }
    double r, x, y, z;
    macros_ref<Q>(a, r, x, y, z);
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double fe = feq_heluo_ref<Q>(k, r, x, y, z);
        cf[k * nc + i] = fe + scale * (a[k] - fe);
    }
}

// Non-equilibrium extrapolation ("eflow stable" form) for one boundary set:
// f_k(b) = feq_k(rho_b, u_bc) + f_k(b + e_k) - feq_k(rho_n, u_n) on the
// reserved directions (NonEquilibrumExtrapolation.cpp:33-71).  Boundary-cell
// f is read by nothing but this update, so it runs as a Jacobi sweep per set
// (values computed first, then written).
__constant__ int8_t c_bdry19[26][14];
__constant__ int8_t c_bdry27[26][18];

template <int Q>
__global__ void k_bc_neq(const int32_t *list, int64_t nl, int b, int64_t n, const int32_t *nbr, const double *rho,
                         const double *u, double *f, double ubx, double uby, double ubz, double *tmp, int phase,
                         int *err)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    constexpr int W = Q == 19 ? 14 : 18;
    for (int t = 0; t < W; ++t) {
        const int k = Q == 19 ? c_bdry19[b][t] : c_bdry27[b][t];
        if (k < 0) break;
        if (phase == 0) {
            const int32_t nb = k == 0 ? (int32_t)i : nbr[(int64_t)(k - 1) * n + i];
            if (nb < 0) {
                atomicOr(err, DEVERR_MISSING_BC_NBR);
                tmp[t * nl + j] = f[k * n + i];
                continue;
            }
            const double fw = feq_ref<Q>(k, rho[i], ubx, uby, ubz);
            const double fn = feq_ref<Q>(k, rho[nb], u[nb], u[n + nb], u[2 * n + nb]);
            tmp[t * nl + j] = fw + f[k * n + nb] - fn;
        } else {
            f[k * n + i] = tmp[t * nl + j];
        }
    }
}

// Restated inlet/outflow on the x faces: West wall cells hold
// fcol = feq(rho_inner, u_bc), East wall cells copy the inner cell's fcol.
template <int Q>
__global__ void k_bc_inout(const int32_t *list, int64_t nl, int east, int64_t n, const int32_t *nbr, const double *rho,
                           double *f, double *fcol, double ubx, double uby, double ubz, int *err)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    const int32_t nb = nbr[(int64_t)((east ? 2 : 1) - 1) * n + i];
    if (nb < 0) {
        atomicOr(err, DEVERR_MISSING_BC_NBR);
        return;
    }
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double v = east ? fcol[k * n + nb] : feq_ref<Q>(k, rho[nb], ubx, uby, ubz);
        fcol[k * n + i] = v;
        f[k * n + i] = v;
    }
}

// SinglePointInterpolation::treat (ComplexBoundary_Manager.cpp:43-225):
// wall links by Filippova-Haenel or distance-weighted interpolation, free
// links by plain pull, density clamp, eight multi-direct-forcing sweeps (each
// cell only touches its own populations, so the sweeps run in registers).
template <int Q, int FH>
__global__ void k_ib_treat(const int32_t *list, int64_t nl, int64_t n, const int32_t *disrow, const double *dis,
                           const int32_t *nbr, const double *fcol, const double *rho, double *f, double *force)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    const double *dr = dis + (int64_t)disrow[i] * (Q - 1);
    const double rho_b = rho[i];
    double g[Q];
    g[0] = fcol[i];
    double fx = 0., fy = 0., fz = 0.;
#pragma unroll
    for (int k = 1; k < Q; ++k) {
        const double dd = dr[inv(k) - 1];
        if (dd != -1.) {
            const double finc = fcol[inv(k) * n + i];
            const int32_t si = nbr[(int64_t)(inv(k) - 1) * n + i];
            const double fstr = si >= 0 ? fcol[k * n + si] : finc;
            double fnew;
            if (FH) {
                if (dd < 0.5) {
                    fnew = (1.0 - 2.0 * dd) * finc + 2.0 * dd * fstr;
                } else {
                    const double feqw = w19z(inv(k)) * rho_b;
                    const double inv2d = 1.0 / (2.0 * dd);
                    fnew = inv2d * fstr + (1.0 - inv2d) * feqw;
                }
            } else {
                fnew = (1.0 - dd) * finc + dd * fstr;
            }
            g[k] = fnew;
            const double mt = finc + fnew;
            fx += -mt * ex(k);
            fy += -mt * ey(k);
            fz += -mt * ez(k);
        } else {
            const int32_t si = nbr[(int64_t)(k - 1) * n + i];
            g[k] = si < 0 ? fcol[inv(k) * n + i] : fcol[k * n + si];
        }
    }
    double ra = 0.;
#pragma unroll
    for (int k = 0; k < Q; ++k) ra += g[k];
    if (ra < 0.3)
        g[0] += 1.0 * (0.3 - ra);
    else if (ra < 0.5)
        g[0] += 0.5 * (0.5 - ra);
    else if (ra > 3.0)
        g[0] += 1.0 * (3.0 - ra);
    else if (ra > 2.0)
        g[0] += 0.5 * (2.0 - ra);
    for (int it = 0; it < 8; ++it) {
        double r = 0., ux = 0., uy = 0., uz = 0.;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            r += g[k];
            ux += g[k] * ex(k);
            uy += g[k] * ey(k);
            uz += g[k] * ez(k);
        }
        if (r <= 0.) continue;
        ux = ux / r;
        uy = uy / r;
        uz = uz / r;
        const double um = sqrt(ux * ux + uy * uy + uz * uz);
        if (um < 1e-10) continue;
        const double mx = -0.5 * r * ux, my = -0.5 * r * uy, mz = -0.5 * r * uz;
        double adj = 0.;
#pragma unroll
        for (int k = 1; k < Q; ++k) {
            if (dr[inv(k) - 1] == -1.) continue;
            const double df = w19z(k) * 3.0 * (ex(k) * mx + ey(k) * my + ez(k) * mz);
            g[k] += df;
            adj -= df;
        }
        g[0] += adj;
    }
#pragma unroll
    for (int k = 0; k < Q; ++k) f[k * n + i] = g[k];
    force[j] = fx;
    force[nl + j] = fy;
    force[2 * nl + j] = fz;
}

// fixed-order reduction of the per-cell IB force into the accumulator
// (LBM_Manager::accumIBForce, one call per treat)
__global__ void k_force_reduce(const double *force, int64_t nl, double *acc)
{
    __shared__ double s[3][256];
    const int t = threadIdx.x;
    double a[3] = {0., 0., 0.};
    for (int64_t j = t; j < nl; j += blockDim.x)
        for (int c = 0; c < 3; ++c) a[c] += force[c * nl + j];
    for (int c = 0; c < 3; ++c) s[c][t] = a[c];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (t < w)
            for (int c = 0; c < 3; ++c) s[c][t] += s[c][t + w];
        __syncthreads();
    }
    if (t == 0) {
        for (int c = 0; c < 3; ++c) acc[c] += s[c][0];
        acc[3] += 1.0;
    }
}

__global__ void k_force_tick(double *acc) { acc[3] += 1.0; }

// ----------------------------------------------------------------------------
// host drivers
// ----------------------------------------------------------------------------
static bool g_bdry_uploaded = false;

static int upload_bdry(Ctx &ctx)
{
    if (g_bdry_uploaded) return MT_OK;
    static const int8_t b19[26][14] = {
        {0, 1, 3, 4, 5, 6, 7, 9, 11, 13, 15, 16, 17, 18}, {0, 2, 3, 4, 5, 6, 8, 10, 12, 14, 15, 16, 17, 18},
        {0, 1, 2, 3, 5, 6, 7, 10, 11, 12, 13, 14, 15, 17}, {0, 1, 2, 4, 5, 6, 8, 9, 11, 12, 13, 14, 16, 18},
        {0, 1, 2, 3, 4, 5, 7, 8, 9, 10, 11, 14, 15, 18}, {0, 1, 2, 3, 4, 6, 7, 8, 9, 10, 12, 13, 16, 17},
        {0, 2, 4, 5, 6, 8, 12, 14, 16, 18, -1, -1, -1, -1}, {0, 1, 4, 5, 6, 9, 11, 13, 16, 18, -1, -1, -1, -1},
        {0, 1, 3, 5, 6, 7, 11, 13, 15, 17, -1, -1, -1, -1}, {0, 2, 3, 5, 6, 10, 12, 14, 15, 17, -1, -1, -1, -1},
        {0, 1, 2, 4, 6, 8, 9, 12, 13, 16, -1, -1, -1, -1}, {0, 1, 2, 3, 6, 7, 10, 12, 13, 17, -1, -1, -1, -1},
        {0, 1, 2, 4, 5, 8, 9, 11, 14, 18, -1, -1, -1, -1}, {0, 1, 2, 3, 5, 7, 10, 11, 14, 15, -1, -1, -1, -1},
        {0, 2, 3, 4, 6, 8, 10, 12, 16, 17, -1, -1, -1, -1}, {0, 1, 3, 4, 6, 7, 9, 13, 16, 17, -1, -1, -1, -1},
        {0, 2, 3, 4, 5, 8, 10, 14, 15, 18, -1, -1, -1, -1}, {0, 1, 3, 4, 5, 7, 9, 11, 15, 18, -1, -1, -1, -1},
        {0, 2, 4, 6, 8, 12, 16, -1, -1, -1, -1, -1, -1, -1}, {0, 1, 4, 6, 9, 13, 16, -1, -1, -1, -1, -1, -1, -1},
        {0, 1, 3, 6, 7, 13, 17, -1, -1, -1, -1, -1, -1, -1}, {0, 2, 3, 6, 10, 12, 17, -1, -1, -1, -1, -1, -1, -1},
        {0, 2, 4, 5, 8, 14, 18, -1, -1, -1, -1, -1, -1, -1}, {0, 1, 4, 5, 9, 11, 18, -1, -1, -1, -1, -1, -1, -1},
        {0, 1, 3, 5, 7, 11, 15, -1, -1, -1, -1, -1, -1, -1}, {0, 2, 3, 5, 10, 14, 15, -1, -1, -1, -1, -1, -1, -1}};
    static const int8_t b27[26][18] = {
        {0, 1, 3, 4, 5, 6, 7, 9, 11, 13, 15, 16, 17, 18, 19, 21, 24, 26},
        {0, 2, 3, 4, 5, 6, 8, 10, 12, 14, 15, 16, 17, 18, 20, 22, 23, 25},
        {0, 1, 2, 3, 5, 6, 7, 10, 11, 12, 13, 14, 15, 17, 19, 22, 24, 25},
        {0, 1, 2, 4, 5, 6, 8, 9, 11, 12, 13, 14, 16, 18, 20, 21, 23, 26},
        {0, 1, 2, 3, 4, 5, 7, 8, 9, 10, 11, 14, 15, 18, 19, 21, 23, 25},
        {0, 1, 2, 3, 4, 6, 7, 8, 9, 10, 12, 13, 16, 17, 20, 22, 24, 26},
        {0, 2, 4, 5, 6, 8, 12, 14, 16, 18, 20, 23, -1, -1, -1, -1, -1, -1},
        {0, 1, 4, 5, 6, 9, 11, 13, 16, 18, 21, 26, -1, -1, -1, -1, -1, -1},
        {0, 1, 3, 5, 6, 7, 11, 13, 15, 17, 19, 24, -1, -1, -1, -1, -1, -1},
        {0, 2, 3, 5, 6, 10, 12, 14, 15, 17, 22, 25, -1, -1, -1, -1, -1, -1},
        {0, 1, 2, 4, 6, 8, 9, 12, 13, 16, 20, 26, -1, -1, -1, -1, -1, -1},
        {0, 1, 2, 3, 6, 7, 10, 12, 13, 17, 22, 24, -1, -1, -1, -1, -1, -1},
        {0, 1, 2, 4, 5, 8, 9, 11, 14, 18, 21, 23, -1, -1, -1, -1, -1, -1},
        {0, 1, 2, 3, 5, 7, 10, 11, 14, 15, 19, 25, -1, -1, -1, -1, -1, -1},
        {0, 2, 3, 4, 6, 8, 10, 12, 16, 17, 20, 22, -1, -1, -1, -1, -1, -1},
        {0, 1, 3, 4, 6, 7, 9, 13, 16, 17, 24, 26, -1, -1, -1, -1, -1, -1},
        {0, 2, 3, 4, 5, 8, 10, 14, 15, 18, 23, 25, -1, -1, -1, -1, -1, -1},
        {0, 1, 3, 4, 5, 7, 9, 11, 15, 18, 19, 21, -1, -1, -1, -1, -1, -1},
        {0, 2, 4, 6, 8, 12, 16, 20, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
        {0, 1, 4, 6, 9, 13, 16, 26, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
        {0, 1, 3, 6, 7, 13, 17, 24, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
        {0, 2, 3, 6, 10, 12, 17, 22, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
        {0, 2, 4, 5, 8, 14, 18, 23, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
        {0, 1, 4, 5, 9, 11, 18, 21, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
        {0, 1, 3, 5, 7, 11, 15, 19, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1},
        {0, 2, 3, 5, 10, 14, 15, 25, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1}};
    MT_CUDA(ctx, cudaMemcpyToSymbol(c_bdry19, b19, sizeof(b19)));
    MT_CUDA(ctx, cudaMemcpyToSymbol(c_bdry27, b27, sizeof(b27)));
    g_bdry_uploaded = true;
    return MT_OK;
}

int amr_init_equilibrium(Ctx &ctx, Case &c, double rho0, const double *u0)
{
    for (int l = 0; l <= c.d.max_level; ++l) {
        Level &lv = c.lv[l];
        if (!lv.n) continue;
        if (c.d.q == 19)
            k_init_eq<19><<<grid_for(lv.n, 256), 256, 0, ctx.stream>>>(lv.n, lv.tag, rho0, u0[0], u0[1], u0[2], lv.f,
                                                                        lv.fcol, lv.rho, lv.u);
        else
            k_init_eq<27><<<grid_for(lv.n, 256), 256, 0, ctx.stream>>>(lv.n, lv.tag, rho0, u0[0], u0[1], u0[2], lv.f,
                                                                        lv.fcol, lv.rho, lv.u);
        MT_LAUNCHED(ctx);
    }
    return MT_OK;
}

enum { PH_MACROS = 0, PH_COLLIDE, PH_STREAM, PH_EXPLOSION, PH_COALESCENCE, PH_BC, PH_IB, PH_BC_INOUT,
       PH_BC_FACE0 = 8 };

template <int Q>
static int phase_q(Ctx &ctx, Case &c, int phase, int l)
{
    const int B = 128;
    cudaStream_t s = ctx.stream;
    Level &lv = c.lv[l];
    const int64_t n = lv.n;
    switch (phase) {
    case PH_MACROS:
        if (lv.ncollide) {
            k_macros<Q><<<grid_for(lv.ncollide, B), B, 0, s>>>(lv.collide_list, lv.ncollide, n, lv.f, lv.rho, lv.u);
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    case PH_COLLIDE:
        if (lv.ncollide) {
            if (c.d.collision == MT_COLL_LBGK) {
                k_collide<Q, MT_COLL_LBGK><<<grid_for(lv.ncollide, B), B, 0, s>>>(lv.collide_list, lv.ncollide, n,
                                                                                   c.d.tau[l], lv.f, lv.rho, lv.u,
                                                                                   lv.fcol);
            } else {
                // the cumulant model exists for D3Q27 only (checked at case creation)
                if constexpr (Q == 27)
                    k_collide<Q, MT_COLL_CUMULANT><<<grid_for(lv.ncollide, 64), 64, 0, s>>>(
                        lv.collide_list, lv.ncollide, n, c.d.tau[l], lv.f, lv.rho, lv.u, lv.fcol);
            }
            MT_LAUNCHED(ctx);
        }
        if (lv.nlist[2]) {
            k_copy_fcol<Q><<<grid_for(lv.nlist[2], B), B, 0, s>>>(lv.list[2], lv.nlist[2], n, lv.f, lv.fcol);
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    case PH_STREAM:
        if (lv.nstream) {
            k_stream<Q><<<grid_for(lv.nstream, B), B, 0, s>>>(lv.stream_list, lv.nstream, n, c.d.stream_convention,
                                                               lv.nbr, lv.fcol, lv.f);
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    case PH_EXPLOSION: {
        if (l < 1 || !lv.nexpl) return MT_OK;
        Level &cl = c.lv[l - 1];
        const double scale = (2.0 * c.d.tau[l]) / c.d.tau[l - 1];
        k_explosion<Q><<<grid_for(lv.nexpl, B), B, 0, s>>>(lv.expl_src, lv.expl_child, lv.nexpl, cl.n, cl.fcol, n,
                                                            lv.fcol, scale);
        MT_LAUNCHED(ctx);
        return MT_OK;
    }
    case PH_COALESCENCE: {
        if (l >= c.d.max_level || !lv.nlist[1]) return MT_OK;
        Level &fl = c.lv[l + 1];
        const double scale = c.d.tau[l] / (2.0 * c.d.tau[l + 1]);
        k_coalescence<Q><<<grid_for(lv.nlist[1], B), B, 0, s>>>(lv.list[1], lv.coal_child, lv.nlist[1], n, lv.f,
                                                                 fl.f, fl.n, scale);
        MT_LAUNCHED(ctx);
        return MT_OK;
    }
    case PH_BC:
    case PH_BC_FACE0 + 0: case PH_BC_FACE0 + 1: case PH_BC_FACE0 + 2:
    case PH_BC_FACE0 + 3: case PH_BC_FACE0 + 4: case PH_BC_FACE0 + 5: {
        // all six face groups in the reference's order, or one of them
        const int f0 = phase == PH_BC ? 0 : phase - PH_BC_FACE0, f1 = phase == PH_BC ? 6 : f0 + 1;
        Level &l0 = c.lv[0];
        static const int face_sets[6][9] = {
            {0, 7, 8, 15, 17, 19, 20, 23, 24}, {1, 6, 9, 14, 16, 18, 21, 22, 25},
            {2, 11, 13, -1, -1, -1, -1, -1, -1}, {3, 10, 12, -1, -1, -1, -1, -1, -1},
            {4, -1, -1, -1, -1, -1, -1, -1, -1}, {5, -1, -1, -1, -1, -1, -1, -1, -1}};
        double *tmp = c.bc_tmp;
        if (!tmp) return MT_OK;
        for (int face = f0; face < f1; ++face)
            for (int g = 0; g < 9; ++g) {
                const int b = face_sets[face][g];
                if (b < 0) break;
                if (!l0.nbc[b]) continue;
                for (int ph = 0; ph < 2; ++ph) {
                    k_bc_neq<Q><<<grid_for(l0.nbc[b], B), B, 0, s>>>(l0.bclist[b], l0.nbc[b], b, l0.n, l0.nbr, l0.rho,
                                                                      l0.u, l0.f, c.d.u_bc[0], c.d.u_bc[1],
                                                                      c.d.u_bc[2], tmp, ph, c.dev_err);
                    MT_LAUNCHED(ctx);
                }
            }
        return MT_OK;
    }
    case PH_BC_INOUT: {
        Level &l0 = c.lv[0];
        for (int face = 0; face < 2; ++face) {
            if (!l0.nbc[face]) continue;
            k_bc_inout<Q><<<grid_for(l0.nbc[face], B), B, 0, s>>>(l0.bclist[face], l0.nbc[face], face, l0.n, l0.nbr,
                                                                   l0.rho, l0.f, l0.fcol, c.d.u_bc[0], c.d.u_bc[1],
                                                                   c.d.u_bc[2], c.dev_err);
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    }
    case PH_IB: {
        Level &fl = c.lv[c.d.max_level];
        if (!fl.nib) {
            k_force_tick<<<1, 1, 0, s>>>(c.force_acc);
            MT_LAUNCHED(ctx);
            return MT_OK;
        }
        if (c.d.ib_method == MT_IB_FH)
            k_ib_treat<Q, 1><<<grid_for(fl.nib, 64), 64, 0, s>>>(fl.iblist, fl.nib, fl.n, fl.disrow, c.dis, fl.nbr,
                                                                  fl.fcol, fl.rho, fl.f, c.ib_force);
        else
            k_ib_treat<Q, 0><<<grid_for(fl.nib, 64), 64, 0, s>>>(fl.iblist, fl.nib, fl.n, fl.disrow, c.dis, fl.nbr,
                                                                  fl.fcol, fl.rho, fl.f, c.ib_force);
        MT_LAUNCHED(ctx);
        k_force_reduce<<<1, 256, 0, s>>>(c.ib_force, fl.nib, c.force_acc);
        MT_LAUNCHED(ctx);
        return MT_OK;
    }
    }
    return set_err(ctx, MT_ERR_ARG, "unknown phase");
}

int amr_phase(Ctx &ctx, Case &c, int phase, int level)
{
    if (level < 0 || level > c.d.max_level) return set_err(ctx, MT_ERR_ARG, "level out of range");
    int rc = upload_bdry(ctx);
    if (rc) return rc;
    return c.d.q == 19 ? phase_q<19>(ctx, c, phase, level) : phase_q<27>(ctx, c, phase, level);
}

// LBM_Manager::LBMkernel (LBM_Simulator.cpp:20-229)
int amr_lbm_kernel(Ctx &ctx, Case &c, int l)
{
    const int L = c.d.max_level;
    int rc;
#define RUN(ph, lev)                              \
    do {                                          \
        if ((rc = amr_phase(ctx, c, (ph), (lev)))) \
            return rc;                            \
    } while (0)
    for (int sub = 0; sub < 2; ++sub) {
        RUN(PH_MACROS, l);
        RUN(PH_COLLIDE, l);
        if (l == 0 && c.d.bc_mode == MT_BC_ZOUHE_OUTFLOW) RUN(PH_BC_INOUT, 0);
        if (l < L)
            if ((rc = amr_lbm_kernel(ctx, c, l + 1))) return rc;
        if (sub == 0 && l > 0) RUN(PH_EXPLOSION, l);
        RUN(PH_STREAM, l);
        if (l == 0) {
            if (c.d.bc_mode == MT_BC_NEQ) RUN(PH_BC, 0);
        } else if (l == L) {
            RUN(PH_IB, L);
        }
        if (l < L) RUN(PH_COALESCENCE, l);
        if (l == 0) break;
    }
#undef RUN
    return MT_OK;
}

static int record_step(Ctx &ctx, Case &c)
{
    int rc = amr_lbm_kernel(ctx, c, 0);
    if (rc) return rc;
    for (int l = 0; l <= c.d.max_level; ++l)
        if ((rc = amr_phase(ctx, c, PH_MACROS, l))) return rc;
    return MT_OK;
}

// n coarse steps replayed from one captured graph (fluidSimulate loop body)
int amr_step(Ctx &ctx, Case &c, int n)
{
    int rc = upload_bdry(ctx);
    if (rc) return rc;
    if (!c.graph) {
        // the neq boundary uses a stream-ordered scratch allocation; capture
        // records it as graph memory nodes
        const int64_t before = ctx.launches;
        cudaGraph_t g;
        MT_CUDA(ctx, cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal));
        rc = record_step(ctx, c);
        cudaGraph_t captured = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx.stream, &captured);
        if (rc) {
            if (captured) cudaGraphDestroy(captured);
            return rc;
        }
        if (e != cudaSuccess) return set_err(ctx, MT_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        g = captured;
        c.graph_launches = ctx.launches - before;
        ctx.launches = before;
        e = cudaGraphInstantiate(&c.graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            c.graph = nullptr;
            return set_err(ctx, MT_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
    }
    for (int s = 0; s < n; ++s) {
        MT_CUDA(ctx, cudaGraphLaunch(c.graph, ctx.stream));
        ctx.launches += c.graph_launches;
    }
    return MT_OK;
}

// non-finite guard over f and fcol of one level: raises DEVERR_NONFINITE
// (the reference only prints NaN diagnostics, LBM_Simulator.cpp:33-41)
__global__ void k_guard(const double *f, const double *fcol, int64_t total, int *err)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool bad = false;
    for (; j < total; j += (int64_t)gridDim.x * blockDim.x) bad |= !isfinite(f[j]) || !isfinite(fcol[j]);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, DEVERR_NONFINITE);
}

int amr_guard(Ctx &ctx, Case &c, int *flags)
{
    MT_CUDA(ctx, cudaMemsetAsync(c.dev_err, 0, sizeof(int), ctx.stream));
    for (int l = 0; l <= c.d.max_level; ++l) {
        Level &lv = c.lv[l];
        if (!lv.n) continue;
        const int64_t total = lv.n * c.d.q;
        k_guard<<<std::min<int64_t>(grid_for(total, 256), 148 * 16), 256, 0, ctx.stream>>>(lv.f, lv.fcol, total,
                                                                                          c.dev_err);
        MT_LAUNCHED(ctx);
    }
    MT_CUDA(ctx, cudaMemcpyAsync(flags, c.dev_err, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}

__global__ void k_find(const uint64_t *key, int64_t n, const uint64_t *q, int64_t nq, int64_t *out)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j < nq) out[j] = find_key(key, n, q[j]);
}

int amr_find(Ctx &ctx, Case &c, int level, const uint64_t *h_keys, int64_t nq, int64_t *h_idx)
{
    if (nq == 0) return MT_OK;
    Level &lv = c.lv[level];
    uint64_t *dq = nullptr;
    int64_t *dout = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&dq, 8 * nq, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&dout, 8 * nq, ctx.stream));
    MT_CUDA(ctx, cudaMemcpyAsync(dq, h_keys, 8 * nq, cudaMemcpyHostToDevice, ctx.stream));
    k_find<<<grid_for(nq, 256), 256, 0, ctx.stream>>>(lv.key, lv.n, dq, nq, dout);
    MT_LAUNCHED(ctx);
    MT_CUDA(ctx, cudaMemcpyAsync(h_idx, dout, 8 * nq, cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    cudaFreeAsync(dq, ctx.stream);
    cudaFreeAsync(dout, ctx.stream);
    return MT_OK;
}

}  // namespace mt
