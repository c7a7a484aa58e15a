// Multi-level path: device build of the Morton-sorted SoA levels and the
// driver of the reference's recursive time step (the phase kernels live in
// mt_amr_phases.cuh, one instantiation per storage type).
//
// Layout per level: cells sorted by Morton key; populations f/fcol as
// [Q][n] in the storage type; nbr as [(Q-1)][n] int32 (index of key + e_k
// or -1); index lists (int32) for each reference set in ascending key order.
#include <cub/cub.cuh>

#include <algorithm>
#include <utility>
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
    } else if (s == MT_SET_IB_BAND) {
        bit = TAG_BAND;
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

// ---- 4x4x4 bricks of a level (fused schedule) --------------------------------
__global__ void k_brick_flags(const uint64_t *key, int64_t n, int shift, int32_t *flag)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    flag[i] = (i == 0 || (key[i] >> shift) != (key[i - 1] >> shift)) ? 1 : 0;
}

// cell index at position h of brick b's 6x6x6 neighbourhood (local
// coordinates h % 6 - 1, h / 6 % 6 - 1, h / 36 - 1), or -1
__global__ void k_brick_halo(int64_t nb, const int32_t *bstart, const unsigned long long *bmask,
                             const int32_t *bnbr, int32_t *halo)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 216 * nb) return;
    const int64_t b = t / 216;
    const int h = (int)(t - 216 * b);
    const int nx = h % 6 - 1, ny = (h / 6) % 6 - 1, nz = h / 36 - 1;
    const int sl = ((nx >> 2) + 1) + 3 * ((ny >> 2) + 1) + 9 * ((nz >> 2) + 1);
    const int ax = nx & 3, ay = ny & 3, az = nz & 3;
    const int mm = (ax & 1) | ((ax & 2) << 2) | ((ay & 1) << 1) | ((ay & 2) << 3) | ((az & 1) << 2) | ((az & 2) << 4);
    const int32_t s = bnbr[27 * b + sl];
    int32_t out = -1;
    if (s >= 0) {
        const unsigned long long nm = bmask[s];
        if ((nm >> mm) & 1ull) out = bstart[s] + __popcll(nm & ((1ull << mm) - 1ull));
    }
    halo[t] = out;
}

// cb = inclusive scan of the flags: brick of cell i is cb[i] - 1
__global__ void k_brick_fill(const uint64_t *key, const uint32_t *tag, int64_t n, int shift, int low,
                             const int32_t *cb, int ib_level, int32_t *bstart, uint64_t *bkey,
                             unsigned long long *bmask, uint8_t *bcls)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t b = cb[i] - 1;
    const int m = (int)((key[i] >> low) & 63);
    if (i == 0 || cb[i] != cb[i - 1]) {
        bstart[b] = (int32_t)i;
        bkey[b] = key[i] >> shift;
    }
    atomicOr(bmask + b, 1ull << m);
    const uint32_t t = tag[i];
    // stream covers lat_f then overlap_C2F, and a C2F cell's fcol = f copy
    // comes after the collision (Collision_Manager.cpp:45-52)
    uint8_t cls = 0;
    if (t & TAG_C2F)
        cls = 2;
    else if ((t & TAG_LATF) && (t & TAG_BAND))
        cls = 4;  // direct-forcing band: stream only, collided after the forcing
    else if ((t & TAG_LATF) && !(ib_level && (t & TAG_IB)))
        cls = 1;
    bcls[64 * b + m] = cls;
}

// cells whose streamed f a coarser level's coalescence reads: stream +
// collide with f stored (class 3)
__global__ void k_brick_mark(const int32_t *child, int64_t count, const int32_t *cb, const uint64_t *key, int low,
                             uint8_t *bcls)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int32_t ci = child[t];
    if (ci < 0) return;
    const int64_t b = cb[ci] - 1;
    const int m = (int)((key[ci] >> low) & 63);
    if (bcls[64 * b + m] == 1) bcls[64 * b + m] = 3;
}

// neighbour bricks: Morton_Assist::find_neighbor applied to the corner cell
// of the brick that faces the offset, then a search of the brick keys
__global__ void k_brick_nbrs(MortonGeom g, int level, const uint64_t *bkey, int64_t nb, int shift, int low,
                             int32_t *bnbr)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 27 * nb) return;
    const int64_t b = t / 27;
    const int s = (int)(t - 27 * b);
    const int dx = s % 3 - 1, dy = (s / 3) % 3 - 1, dz = s / 9 - 1;
    const int lx = dx > 0 ? 3 : 0, ly = dy > 0 ? 3 : 0, lz = dz > 0 ? 3 : 0;
    const uint64_t m = (uint64_t)((lx & 1) | ((lx & 2) << 2) | ((ly & 1) << 1) | ((ly & 2) << 3) | ((lz & 1) << 2) |
                                  ((lz & 2) << 4));
    const uint64_t rep = (bkey[b] << shift) | (m << low);
    const uint64_t nk = find_neighbor(g, rep, level, dx, dy, dz);
    bnbr[t] = (int32_t)find_key(bkey, nb, nk >> shift);
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
struct LatfNotBand {
    const uint32_t *tag;
    __host__ __device__ bool operator()(const int32_t &i) const
    {
        return (tag[i] & TAG_LATF) && !(tag[i] & TAG_BAND);
    }
};
struct LatfNotIb {
    const uint32_t *tag;
    __host__ __device__ bool operator()(const int32_t &i) const
    {
        return (tag[i] & TAG_LATF) && !(tag[i] & TAG_IB);
    }
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
    const bool on_dev = lv.draw_keys != nullptr;
    const int64_t nraw = on_dev ? lv.ndraw : (int64_t)lv.raw_keys.size();
    lv.n = 0;
    if (nraw > 0) {
        uint64_t *d_raw = nullptr, *d_sorted = nullptr;
        uint8_t *d_set = nullptr;
        int *d_num = nullptr;
        if (on_dev) {
            d_raw = lv.draw_keys;
            d_set = lv.draw_set;
            lv.draw_keys = nullptr;
            lv.draw_set = nullptr;
            lv.ndraw = 0;
        } else {
            MT_CUDA(ctx, cudaMallocAsync(&d_raw, 8 * nraw, ctx.stream));
            MT_CUDA(ctx, cudaMallocAsync(&d_set, nraw, ctx.stream));
            MT_CUDA(ctx, cudaMemcpyAsync(d_raw, lv.raw_keys.data(), 8 * nraw, cudaMemcpyHostToDevice, ctx.stream));
            MT_CUDA(ctx, cudaMemcpyAsync(d_set, lv.raw_set.data(), nraw, cudaMemcpyHostToDevice, ctx.stream));
        }
        MT_CUDA(ctx, cudaMallocAsync(&d_sorted, 8 * nraw, ctx.stream));
        MT_CUDA(ctx, cudaMallocAsync(&d_num, sizeof(int), ctx.stream));
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
    {
        int rc = amr_dispatch(c, [&](auto *tag) {
            using S = std::remove_pointer_t<decltype(tag)>;
            return AmrOps<S>::alloc(ctx, c, l);
        });
        if (rc) return rc;
    }
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
    for (int f = 0; f < 6; ++f)
        for (int a = 0; a < 3; ++a) c.face_u[f][a] = c.d.u_bc[a];
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
    if (!c.dis_on_device) c.ndis = (int64_t)c.h_dis_key.size();
    const int W = c.d.q - 1;
    if (c.ndis > 0) {
        if (!c.dis_on_device) {
            MT_CUDA(ctx, cudaMallocAsync(&c.dis_key, 8 * c.ndis, ctx.stream));
            MT_CUDA(ctx, cudaMallocAsync(&c.dis, 8 * c.ndis * W, ctx.stream));
            MT_CUDA(ctx, cudaMemcpyAsync(c.dis_key, c.h_dis_key.data(), 8 * c.ndis, cudaMemcpyHostToDevice,
                                         ctx.stream));
            MT_CUDA(ctx, cudaMemcpyAsync(c.dis, c.h_dis.data(), 8 * c.ndis * W, cudaMemcpyHostToDevice, ctx.stream));
        }
        Level &fl = c.lv[L];
        if (fl.n > 0) {
            k_dis_rows<<<grid_for(fl.n, 256), 256, 0, ctx.stream>>>(fl.key, fl.n, c.dis_key, c.ndis, fl.disrow, fl.tag);
            MT_LAUNCHED(ctx);
        }
        k_dis_check<<<grid_for(c.ndis, 256), 256, 0, ctx.stream>>>(c.dis_key, c.ndis, fl.key, fl.n, c.dev_err);
        MT_LAUNCHED(ctx);
        int rc = select_indices(ctx, fl.n, IbLatf{fl.tag}, &fl.iblist, &fl.nib);
        if (rc) return rc;
        // per-cell forces (3 * nib) and the 256-cell partial sums (3 * ceil(nib / 256))
        if (fl.nib)
            MT_CUDA(ctx, cudaMallocAsync(&c.ib_force, 8 * 3 * (fl.nib + grid_for(fl.nib, 256)), ctx.stream));
    }
    {
        int64_t maxn = 0;
        for (int b = 0; b < 26; ++b) maxn = std::max(maxn, c.lv[0].nbc[b]);
        if (maxn) MT_CUDA(ctx, cudaMallocAsync(&c.bc_tmp, sizeof(double) * 18 * maxn, ctx.stream));
        // the concatenated list of all 26 sets for the one-pass sweep
        int64_t tot = 0;
        for (int b = 0; b < 26; ++b) tot += c.lv[0].nbc[b];
        if (tot) {
            c.nbc_all = tot;
            MT_CUDA(ctx, cudaMallocAsync(&c.bc_all, sizeof(int32_t) * tot, ctx.stream));
            MT_CUDA(ctx, cudaMallocAsync(&c.bc_setb, tot, ctx.stream));
            MT_CUDA(ctx, cudaMallocAsync(&c.bc_tmp_all, sizeof(double) * 18 * tot, ctx.stream));
            int64_t off = 0;
            for (int b = 0; b < 26; ++b) {
                const int64_t nb = c.lv[0].nbc[b];
                if (!nb) continue;
                MT_CUDA(ctx, cudaMemcpyAsync(c.bc_all + off, c.lv[0].bclist[b], sizeof(int32_t) * nb,
                                             cudaMemcpyDeviceToDevice, ctx.stream));
                MT_CUDA(ctx, cudaMemsetAsync(c.bc_setb + off, b, nb, ctx.stream));
                off += nb;
            }
        }
    }
    // direct-forcing band of the finest level and its collide list without the band
    {
        Level &fl = c.lv[L];
        if (fl.n) {
            int rc = select_indices(ctx, fl.n, TagHas{fl.tag, TAG_BAND}, &fl.band, &fl.nband);
            if (rc) return rc;
            if (fl.nband) {
                int32_t *lat = nullptr;
                int64_t nlat = 0;
                rc = select_indices(ctx, fl.n, LatfNotBand{fl.tag}, &lat, &nlat);
                if (rc) return rc;
                rc = concat_lists(ctx, lat, nlat, fl.list[1], fl.nlist[1], &fl.collide_nb, &fl.ncollide_nb);
                cudaFreeAsync(lat, ctx.stream);
                if (rc) return rc;
                MT_CUDA(ctx, cudaMallocAsync(&c.acc, sizeof(long long) * 3 * fl.n, ctx.stream));
                MT_CUDA(ctx, cudaMemsetAsync(c.acc, 0, sizeof(long long) * 3 * fl.n, ctx.stream));
                MT_CUDA(ctx, cudaMallocAsync(&c.tstep, sizeof(long long), ctx.stream));
                MT_CUDA(ctx, cudaMemsetAsync(c.tstep, 0, sizeof(long long), ctx.stream));
            }
        }
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

void amr_drop_fused(Case &c)
{
    for (int p = 0; p < 2; ++p) {
        if (c.fgraph[p]) cudaGraphExecDestroy(c.fgraph[p]);
        c.fgraph[p] = nullptr;
    }
    for (int l = 0; l < kMaxLevels; ++l) {
        Level &lv = c.lv[l];
        void *ptrs[] = {lv.fused_list, lv.bstart, lv.bmask, lv.bnbr, lv.bcls, lv.bhalo};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        lv.fused_list = nullptr;
        lv.nfused = 0;
        lv.bstart = nullptr;
        lv.bmask = nullptr;
        lv.bnbr = nullptr;
        lv.bcls = nullptr;
        lv.bhalo = nullptr;
        lv.nbrick = 0;
        lv.bricks = false;
    }
}

void amr_free(Case &c)
{
    for (int l = 0; l < kMaxLevels; ++l) {
        Level &lv = c.lv[l];
        void *ptrs[] = {lv.key, lv.tag, lv.bcidx, lv.disrow, lv.nbr, lv.f, lv.fcol, lv.rho, lv.u,
                        lv.collide_list, lv.stream_list, lv.iblist, lv.expl_src, lv.expl_child, lv.coal_child,
                        lv.fcol_alt, lv.fused_list, lv.bstart, lv.bmask, lv.bnbr, lv.bcls, lv.bhalo,
                        lv.band, lv.collide_nb, lv.draw_keys, lv.draw_set, lv.expl_prev, lv.info_prev};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        for (int s = 0; s < kNumSets; ++s)
            if (lv.list[s]) cudaFree(lv.list[s]);
        for (int b = 0; b < 26; ++b)
            if (lv.bclist[b]) cudaFree(lv.bclist[b]);
        lv = Level();
    }
    if (c.h_force) cudaFreeHost(c.h_force);
    c.h_force = nullptr;
    void *ptrs[] = {c.dis_key, c.dis, c.ib_force, c.force_acc, c.dev_err, c.bc_tmp, c.bc_all, c.bc_setb, c.bc_tmp_all,
                    c.mref, c.mdv, c.path, c.mforce, c.tstep, c.acc, c.mgrid};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    c.bc_tmp = nullptr;
    c.bc_all = nullptr;
    c.bc_setb = nullptr;
    c.bc_tmp_all = nullptr;
    c.nbc_all = 0;
    c.dis_key = nullptr;
    c.dis = nullptr;
    c.ib_force = nullptr;
    c.force_acc = nullptr;
    c.dev_err = nullptr;
    c.mref = c.mdv = c.path = c.mforce = nullptr;
    c.tstep = nullptr;
    c.acc = nullptr;
    c.mgrid = nullptr;
    c.nm = 0;
    if (c.graph) cudaGraphExecDestroy(c.graph);
    c.graph = nullptr;
    for (int p = 0; p < 2; ++p) {
        if (c.fgraph[p]) cudaGraphExecDestroy(c.fgraph[p]);
        c.fgraph[p] = nullptr;
    }
    if (c.side) cudaStreamDestroy(c.side);
    if (c.ev_fork) cudaEventDestroy(c.ev_fork);
    if (c.ev_join) cudaEventDestroy(c.ev_join);
    c.side = nullptr;
    c.ev_fork = c.ev_join = nullptr;
}

// ----------------------------------------------------------------------------
// driver: the reference's recursion issued as phase kernels of the case's
// storage type (mt_amr_phases.cuh, instantiated in mt_amr_f64.cu and
// mt_amr_lp.cu)
// ----------------------------------------------------------------------------

int amr_phase(Ctx &ctx, Case &c, int phase, int level)
{
    if (level < 0 || level > c.d.max_level) return set_err(ctx, MT_ERR_ARG, "level out of range");
    return amr_dispatch(c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return AmrOps<S>::phase(ctx, c, phase, level);
    });
}

int amr_init_equilibrium(Ctx &ctx, Case &c, double rho0, const double *u0)
{
    c.prev_stale = true;
    return amr_dispatch(c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return AmrOps<S>::init_eq(ctx, c, rho0, u0);
    });
}

// LBM_Manager::LBMkernel (LBM_Simulator.cpp:20-229).  The collision kernel
// computes the macros it needs from the same populations the reference's
// calculateMacros(level) reads just before collide(level), so the separate
// macros pass of each substep is folded into it.
int amr_lbm_kernel(Ctx &ctx, Case &c, int l)
{
    const int L = c.d.max_level;
    int rc;
#define RUN(ph, lev)                               \
    do {                                           \
        if ((rc = amr_phase(ctx, c, (ph), (lev)))) \
            return rc;                             \
    } while (0)
    for (int sub = 0; sub < 2; ++sub) {
        RUN(PH_COLLIDE, l);
        if (l == 0 && c.d.bc_mode == MT_BC_ZOUHE_OUTFLOW) RUN(PH_BC_INOUT, 0);
        if (l < L)
            if ((rc = amr_lbm_kernel(ctx, c, l + 1))) return rc;
        if (l > 0 && sub == 0) RUN(PH_EXPLOSION, l);
        if (l > 0 && sub == 1 && c.itime != MT_ITIME_REFERENCE) RUN(PH_EXPLOSION_B, l);
        RUN(PH_STREAM, l);
        if (l == 0) {
            if (c.d.bc_mode == MT_BC_NEQ) RUN(PH_BC, 0);
            if (c.d.bc_mode == MT_BC_ZOUHE_HH) RUN(PH_BC_HH, 0);
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

static int capture(Ctx &ctx, Case &c, int (*record)(Ctx &, Case &), cudaGraphExec_t *out, int64_t *launches)
{
    const int64_t before = ctx.launches;
    MT_CUDA(ctx, cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal));
    int rc = record(ctx, c);
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx.stream, &captured);
    if (rc) {
        if (captured) cudaGraphDestroy(captured);
        return rc;
    }
    if (e != cudaSuccess) return set_err(ctx, MT_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
    *launches = ctx.launches - before;
    ctx.launches = before;
    e = cudaGraphInstantiate(out, captured, 0);
    cudaGraphDestroy(captured);
    if (e != cudaSuccess) {
        *out = nullptr;
        return set_err(ctx, MT_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    return MT_OK;
}

// ---- fused schedule ---------------------------------------------------------
// Per substep of level l: swap the post-collision buffers (fcol now holds the
// collision computed one substep ahead, F2C cells included), the
// inlet/outflow wall cells, the finer levels, the explosion, then one pass
// that streams lat_f and C2F, treats the IB cells and collides all of them
// into the other buffer for the next substep; then the boundary sweep, and
// coalescence followed by the F2C cells' next collision, as in
// LBM_Simulator.cpp:20-229.  On each level's last substep of the coarse step
// the passes also write the macros of the f they leave (the all-level
// calculateMacros of LBM_Simulator.cpp:11-17), except on level 0 under the
// non-equilibrium boundary, whose sweep reads the substep's earlier macros.
static void swap_buffers(Case &c, int l)
{
    std::swap(c.lv[l].fcol, c.lv[l].fcol_alt);
    if (l == 0) c.par0 ^= 1;
}

static int fused_lbm_kernel(Ctx &ctx, Case &c, int l, bool last_parent)
{
    const int L = c.d.max_level;
    int rc;
#define RUN(ph, lev)                               \
    do {                                           \
        if ((rc = amr_phase(ctx, c, (ph), (lev)))) \
            return rc;                             \
    } while (0)
    for (int sub = 0; sub < 2; ++sub) {
        const bool last = last_parent && (l == 0 || sub == 1);
        swap_buffers(c, l);
        if (l == 0 && c.d.bc_mode == MT_BC_ZOUHE_OUTFLOW) RUN(PH_BC_INOUT, 0);
        if (l < L)
            if ((rc = fused_lbm_kernel(ctx, c, l + 1, last))) return rc;
        if (l > 0 && sub == 0) RUN(PH_EXPLOSION, l);
        if (l > 0 && sub == 1 && c.itime != MT_ITIME_REFERENCE) RUN(PH_EXPLOSION_B, l);
        c.macros_now = last && !(l == 0 && c.d.bc_mode == MT_BC_NEQ);
        RUN(PH_PULL_COLLIDE, l);
        if (l == L && c.lv[l].nband) RUN(PH_DF, l);
        if (l == 0 && c.d.bc_mode == MT_BC_NEQ) RUN(PH_BC, 0);
        if (l < L) RUN(PH_COAL_COLLIDE, l);
        c.macros_now = 0;
        if (l == 0) break;
    }
#undef RUN
    return MT_OK;
}

static int record_fused_step(Ctx &ctx, Case &c)
{
    int rc = fused_lbm_kernel(ctx, c, 0, true);
    if (rc) return rc;
    if (c.d.bc_mode == MT_BC_NEQ)
        if ((rc = amr_phase(ctx, c, PH_MACROS, 0))) return rc;
    return MT_OK;
}

// Bricks of level l, when they reproduce the neighbour table exactly: every
// periodic axis spans a multiple of 4 cells at this level (the wrap then
// falls on a brick boundary).
static int build_bricks(Ctx &ctx, Case &c, int l)
{
    Level &lv = c.lv[l];
    const int L = c.d.max_level;
    for (int a = 0; a < 3; ++a)
        if (c.d.periodic[a] && ((c.d.extent0[a] << l) % 4) != 0) return MT_OK;
    const int64_t n = lv.n;
    if (n * c.d.q >= ((int64_t)1 << 32)) return MT_OK;  // the brick pass uses 32-bit element offsets
    const int low = 3 * (L - l), shift = low + 6;
    int32_t *flag = nullptr, *cb = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&flag, 4 * n, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&cb, 4 * n, ctx.stream));
    k_brick_flags<<<grid_for(n, 256), 256, 0, ctx.stream>>>(lv.key, n, shift, flag);
    MT_LAUNCHED(ctx);
    size_t tb = 0;
    MT_CUDA(ctx, cub::DeviceScan::InclusiveSum(nullptr, tb, flag, cb, (int)n, ctx.stream));
    void *tmp = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&tmp, tb, ctx.stream));
    MT_CUDA(ctx, cub::DeviceScan::InclusiveSum(tmp, tb, flag, cb, (int)n, ctx.stream));
    int32_t nb = 0;
    MT_CUDA(ctx, cudaMemcpyAsync(&nb, cb + (n - 1), 4, cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    uint64_t *bkey = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&lv.bstart, 4 * (size_t)nb, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&lv.bmask, 8 * (size_t)nb, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&lv.bnbr, 4 * 27 * (size_t)nb, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&lv.bcls, 64 * (size_t)nb, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&bkey, 8 * (size_t)nb, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.bmask, 0, 8 * (size_t)nb, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.bcls, 0, 64 * (size_t)nb, ctx.stream));
    const int ib_level = (l == L && l > 0) ? 1 : 0;
    k_brick_fill<<<grid_for(n, 256), 256, 0, ctx.stream>>>(lv.key, lv.tag, n, shift, low, cb, ib_level, lv.bstart,
                                                           bkey, (unsigned long long *)lv.bmask, lv.bcls);
    MT_LAUNCHED(ctx);
    if (l > 0 && c.lv[l - 1].coal_child && c.lv[l - 1].nlist[1]) {
        const int64_t cnt = 8 * c.lv[l - 1].nlist[1];
        k_brick_mark<<<grid_for(cnt, 256), 256, 0, ctx.stream>>>(c.lv[l - 1].coal_child, cnt, cb, lv.key, low,
                                                                 lv.bcls);
        MT_LAUNCHED(ctx);
    }
    k_brick_nbrs<<<grid_for(27 * (int64_t)nb, 256), 256, 0, ctx.stream>>>(c.geom, l, bkey, nb, shift, low, lv.bnbr);
    MT_LAUNCHED(ctx);
    MT_CUDA(ctx, cudaMallocAsync(&lv.bhalo, 4 * 216 * (size_t)nb, ctx.stream));
    k_brick_halo<<<grid_for(216 * (int64_t)nb, 256), 256, 0, ctx.stream>>>(nb, lv.bstart,
                                                                          (const unsigned long long *)lv.bmask,
                                                                          lv.bnbr, lv.bhalo);
    MT_LAUNCHED(ctx);
    cudaFreeAsync(tmp, ctx.stream);
    cudaFreeAsync(flag, ctx.stream);
    cudaFreeAsync(cb, ctx.stream);
    cudaFreeAsync(bkey, ctx.stream);
    lv.nbrick = nb;
    lv.bricks = true;
    return MT_OK;
}

// second buffers, the fused cell lists, and the lookahead collision of the
// current f on every level
static int prime_fused(Ctx &ctx, Case &c)
{
    const int L = c.d.max_level;
    if (!c.side && L > 0 && c.lv[L].nib) {
        MT_CUDA(ctx, cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking));
        MT_CUDA(ctx, cudaEventCreateWithFlags(&c.ev_fork, cudaEventDisableTiming));
        MT_CUDA(ctx, cudaEventCreateWithFlags(&c.ev_join, cudaEventDisableTiming));
    }
    for (int l = 0; l <= L; ++l) {
        Level &lv = c.lv[l];
        if (!lv.n) continue;
        if (!lv.fcol_alt) {
            const size_t bytes = (size_t)c.d.q * (size_t)lv.n *
                                 (c.d.storage == MT_STORE_F64 ? 8 : c.d.storage == MT_STORE_F32 ? 4 : 2);
            MT_CUDA(ctx, cudaMallocAsync(&lv.fcol_alt, bytes, ctx.stream));
        }
        if (!lv.bricks && c.use_bricks) {
            int rc = build_bricks(ctx, c, l);
            if (rc) return rc;
        }
        if (!lv.bricks && !lv.fused_list && lv.nlist[0]) {
            int rc = lv.nband ? select_indices(ctx, lv.n, LatfNotBand{lv.tag}, &lv.fused_list, &lv.nfused)
                     : (l == L && l > 0) ? select_indices(ctx, lv.n, LatfNotIb{lv.tag}, &lv.fused_list, &lv.nfused)
                                         : select_indices(ctx, lv.n, TagHas{lv.tag, TAG_LATF}, &lv.fused_list,
                                                          &lv.nfused);
            if (rc) return rc;
        }
        int rc = amr_phase(ctx, c, PH_PRIME, l);
        if (rc) return rc;
    }
    c.primed = true;
    return MT_OK;
}

// the streamed f the fused passes left unstored (class-1 brick cells), for
// every reader outside the fused schedule
int amr_sync_f(Ctx &ctx, Case &c)
{
    if (!c.f_stale) return MT_OK;
    for (int l = 0; l <= c.d.max_level; ++l) {
        int rc = amr_phase(ctx, c, PH_SYNC_F, l);
        if (rc) return rc;
    }
    c.f_stale = false;
    return MT_OK;
}

// a face strategy's velocity: its boundary cells restart from feq(rho0, u)
// and its non-equilibrium sweep (or the West inlet) uses u from now on
int amr_set_face(Ctx &ctx, Case &c, int face, const double *u)
{
    if (int rc = amr_sync_f(ctx, c)) return rc;
    for (int a = 0; a < 3; ++a) c.face_u[face][a] = u[a];
    if (c.graph) cudaGraphExecDestroy(c.graph);
    c.graph = nullptr;
    for (int p = 0; p < 2; ++p) {
        if (c.fgraph[p]) cudaGraphExecDestroy(c.fgraph[p]);
        c.fgraph[p] = nullptr;
    }
    c.primed = false;
    return amr_phase(ctx, c, PH_FACE_EQ0 + face, 0);
}

// n coarse steps replayed from one captured graph (fluidSimulate loop body)
int amr_prev_sync(Ctx &ctx, Case &c)
{
    if (c.itime != MT_ITIME_EXTRAP) return MT_OK;
    const size_t sb = c.d.storage == MT_STORE_F64 ? 8 : c.d.storage == MT_STORE_F32 ? 4 : 2;
    for (int l = 1; l <= c.d.max_level; ++l) {
        Level &lv = c.lv[l];
        if (!lv.nexpl || lv.expl_prev) continue;
        MT_CUDA(ctx, cudaMallocAsync(&lv.expl_prev, sb * (size_t)c.d.q * (size_t)lv.nexpl, ctx.stream));
        c.prev_stale = true;
    }
    if (!c.prev_stale) return MT_OK;
    for (int l = 1; l <= c.d.max_level; ++l)
        if (int rc = amr_phase(ctx, c, PH_EXPL_SAVE, l)) return rc;
    c.prev_stale = false;
    return MT_OK;
}

int amr_step(Ctx &ctx, Case &c, int n)
{
    int rc;
    if ((rc = amr_prev_sync(ctx, c))) return rc;
    if (c.schedule == MT_SCHED_FUSED) {
        if (!c.primed && (rc = prime_fused(ctx, c))) return rc;
        for (int s = 0; s < n; ++s) {
            const int p = c.par0;
            if (!c.fgraph[p]) {
                // recording swaps the host-side buffer pointers exactly as one
                // replay does, so after it the state matches a launched step
                if ((rc = capture(ctx, c, record_fused_step, &c.fgraph[p], &c.fgraph_launches[p]))) {
                    c.primed = false;
                    return rc;
                }
            } else {
                // the host-side effect of one replay: level 0 swaps once,
                // levels >= 1 an even number of times
                swap_buffers(c, 0);
            }
            MT_CUDA(ctx, cudaGraphLaunch(c.fgraph[p], ctx.stream));
            ctx.launches += c.fgraph_launches[p];
            for (int l = 0; l <= c.d.max_level; ++l) c.f_stale |= c.lv[l].bricks;
        }
        return MT_OK;
    }
    if ((rc = amr_sync_f(ctx, c))) return rc;
    c.primed = false;
    if (c.graph && c.graph_par0 != c.par0) {
        cudaGraphExecDestroy(c.graph);
        c.graph = nullptr;
    }
    if (!c.graph) {
        if ((rc = capture(ctx, c, record_step, &c.graph, &c.graph_launches))) return rc;
        c.graph_par0 = c.par0;
    }
    for (int s = 0; s < n; ++s) {
        MT_CUDA(ctx, cudaGraphLaunch(c.graph, ctx.stream));
        ctx.launches += c.graph_launches;
    }
    return MT_OK;
}

int amr_prime(Ctx &ctx, Case &c)
{
    return c.primed ? MT_OK : prime_fused(ctx, c);
}

// ---- batches ------------------------------------------------------------------
// Every member takes the fused schedule's steps in lockstep: the recursion
// below visits each level with all members that have it, in the order each
// member alone would take (members never interact, so this is the same
// computation as stepping them one by one).  The streamed + collided pass
// of brick levels is one batched kernel per model family; a member's other
// phases run on a pool of streams (parallel graph branches).
namespace {

struct BatchRec {
    Batch *b;
    std::vector<BrickBatch> *hdesc;
    BrickBatch *dbase = nullptr;
    int64_t cap = 0;
};

template <class Pred, class F>
int fork_cases(Ctx &ctx, BatchRec &R, const std::vector<Case *> &cs, Pred &&has, F &&fn)
{
    std::vector<Case *> work;
    for (Case *c : cs)
        if (has(*c)) work.push_back(c);
    if (work.empty()) return MT_OK;
    Batch &B = *R.b;
    cudaStream_t main = ctx.stream;
    const int P = (int)std::min<size_t>(B.pool.size(), work.size());
    MT_CUDA(ctx, cudaEventRecord(B.ev_fork, main));
    for (int p = 0; p < P; ++p) MT_CUDA(ctx, cudaStreamWaitEvent(B.pool[p], B.ev_fork, 0));
    int rc = MT_OK;
    for (size_t i = 0; i < work.size() && !rc; ++i) {
        ctx.stream = B.pool[i % P];
        rc = fn(*work[i]);
    }
    ctx.stream = main;
    for (int p = 0; p < P; ++p) {
        MT_CUDA(ctx, cudaEventRecord(B.ev_join[p], B.pool[p]));
        MT_CUDA(ctx, cudaStreamWaitEvent(main, B.ev_join[p], 0));
    }
    return rc;
}

int storage_code(const Case &c) { return c.d.storage; }

// batched brick passes of level l over the members in cs (brick levels only)
int batch_bricks(Ctx &ctx, BatchRec &R, const std::vector<Case *> &cs, int l, const BrickBatch **first_desc)
{
    // group by (q, collision, storage, storage shift): one kernel instantiation
    // each, the shift a parameter of the pass
    auto same_shift = [l](const Case &a, const Case &b) {
        for (int k = 0; k < 27; ++k)
            if (a.shift[l].d[k] != b.shift[l].d[k]) return false;
        return true;
    };
    std::vector<std::vector<Case *>> groups;
    for (Case *c : cs) {
        if (!c->lv[l].bricks || c->lv[l].nbrick >= kBatchOwnBricks) continue;
        bool placed = false;
        for (auto &g : groups)
            if (g[0]->d.q == c->d.q && g[0]->d.collision == c->d.collision &&
                storage_code(*g[0]) == storage_code(*c) && same_shift(*g[0], *c)) {
                g.push_back(c);
                placed = true;
                break;
            }
        if (!placed) groups.push_back({c});
    }
    (void)first_desc;
    for (auto &g : groups) {
        for (size_t c0 = 0; c0 < g.size(); c0 += kMaxBatchSlots) {
            if ((int64_t)R.hdesc->size() >= R.cap) return set_err(ctx, MT_ERR_STATE, "batch descriptor capacity");
            BrickBatch d;
            const size_t c1 = std::min(g.size(), c0 + kMaxBatchSlots);
            for (size_t k = c0; k < c1; ++k) {
                Case &c = *g[k];
                Level &lv = c.lv[l];
                BrickSlot &sl = d.slot[d.nslots];
                sl.halo = lv.bhalo;
                sl.cls = lv.bcls;
                sl.fcol = lv.fcol;
                sl.f = lv.f;
                sl.fnext = lv.fcol_alt;
                sl.rho = lv.rho;
                sl.u = lv.u;
                sl.tau = c.d.tau[l];
                sl.n = (uint32_t)lv.n;
                sl.textbook = c.d.stream_convention;
                sl.fall = (l == 0 && c.d.bc_mode == MT_BC_NEQ) ? 1 : 0;
                sl.macros = c.macros_now;
                sl.acc = (l == c.d.max_level && lv.nband) ? c.acc : nullptr;
                d.off[d.nslots + 1] = d.off[d.nslots] + lv.nbrick;
                ++d.nslots;
            }
            d.total = d.off[d.nslots];
            const BrickBatch *dev = R.dbase + R.hdesc->size();
            R.hdesc->push_back(d);
            Case &c = *g[0];
            int rc = amr_dispatch(c, [&](auto *tag) {
                using S = std::remove_pointer_t<decltype(tag)>;
                return AmrOps<S>::batch_pass(ctx, c.d.q, c.d.collision, dev, d.total, c.shift[l]);
            });
            if (rc) return rc;
        }
    }
    return MT_OK;
}

int batch_lbm_kernel(Ctx &ctx, BatchRec &R, const std::vector<Case *> &all, int l, bool last_parent)
{
    std::vector<Case *> cs;
    for (Case *c : all)
        if (c->d.max_level >= l && c->lv[l].n) cs.push_back(c);
    if (cs.empty()) return MT_OK;
    int rc;
    for (int sub = 0; sub < 2; ++sub) {
        const bool last = last_parent && (l == 0 || sub == 1);
        for (Case *c : cs) swap_buffers(*c, l);
        if (l == 0)
            if ((rc = fork_cases(ctx, R, cs, [](Case &c) { return c.d.bc_mode == MT_BC_ZOUHE_OUTFLOW; },
                                 [&](Case &c) { return amr_phase(ctx, c, PH_BC_INOUT, 0); })))
                return rc;
        if ((rc = batch_lbm_kernel(ctx, R, cs, l + 1, last))) return rc;
        if (l > 0)
            if ((rc = fork_cases(ctx, R, cs, [sub](Case &c) { return sub == 0 || c.itime != MT_ITIME_REFERENCE; },
                                 [&](Case &c) { return amr_phase(ctx, c, sub == 0 ? PH_EXPLOSION : PH_EXPLOSION_B, l); })))
                return rc;
        for (Case *c : cs) c->macros_now = last && !(l == 0 && c->d.bc_mode == MT_BC_NEQ);
        // members' own pull work (IB cells; levels without bricks; levels
        // large enough to fill the GPU alone) beside the batched brick pass
        {
            Batch &B = *R.b;
            cudaStream_t main = ctx.stream;
            std::vector<Case *> own;
            auto batched = [&](const Case *c) { return c->lv[l].bricks && c->lv[l].nbrick < kBatchOwnBricks; };
            for (Case *c : cs)
                if (!batched(c) || (l == c->d.max_level && l > 0)) own.push_back(c);
            const int P = (int)std::min<size_t>(B.pool.size(), own.size());
            if (P) {
                MT_CUDA(ctx, cudaEventRecord(B.ev_fork, main));
                for (int p = 0; p < P; ++p) MT_CUDA(ctx, cudaStreamWaitEvent(B.pool[p], B.ev_fork, 0));
                for (size_t i = 0; i < own.size(); ++i) {
                    Case &c = *own[i];
                    ctx.stream = B.pool[i % P];
                    c.pull_mode = batched(&c) ? 1 : 0;
                    rc = amr_phase(ctx, c, PH_PULL_COLLIDE, l);
                    c.pull_mode = 0;
                    if (rc) {
                        ctx.stream = main;
                        return rc;
                    }
                }
                ctx.stream = main;
            }
            if ((rc = batch_bricks(ctx, R, cs, l, nullptr))) return rc;
            for (int p = 0; p < P; ++p) {
                MT_CUDA(ctx, cudaEventRecord(B.ev_join[p], B.pool[p]));
                MT_CUDA(ctx, cudaStreamWaitEvent(main, B.ev_join[p], 0));
            }
        }
        if ((rc = fork_cases(ctx, R, cs, [&](Case &c) { return l == c.d.max_level && c.lv[l].nband > 0; },
                             [&](Case &c) { return amr_phase(ctx, c, PH_DF, l); })))
            return rc;
        if ((rc = fork_cases(ctx, R, cs,
                             [&](Case &c) { return (l == 0 && c.d.bc_mode == MT_BC_NEQ) || l < c.d.max_level; },
                             [&](Case &c) {
                                 int r = MT_OK;
                                 if (l == 0 && c.d.bc_mode == MT_BC_NEQ) r = amr_phase(ctx, c, PH_BC, 0);
                                 if (!r && l < c.d.max_level) r = amr_phase(ctx, c, PH_COAL_COLLIDE, l);
                                 return r;
                             })))
            return rc;
        for (Case *c : cs) c->macros_now = 0;
        if (l == 0) break;
    }
    return MT_OK;
}

int record_batch_step(Ctx &ctx, BatchRec &R, const std::vector<Case *> &cases)
{
    int rc = batch_lbm_kernel(ctx, R, cases, 0, true);
    if (rc) return rc;
    return fork_cases(ctx, R, cases, [](Case &c) { return c.d.bc_mode == MT_BC_NEQ; },
                      [&](Case &c) { return amr_phase(ctx, c, PH_MACROS, 0); });
}

}  // namespace

void batch_drop(Batch &b)
{
    for (int p = 0; p < 3; ++p) {
        if (b.graph[p]) cudaGraphExecDestroy(b.graph[p]);
        b.graph[p] = nullptr;
        // stream-ordered: no device-wide synchronisation on a membership change
        if (b.ddesc[p]) cudaFreeAsync(b.ddesc[p], b.free_stream);
        b.ddesc[p] = nullptr;
        b.hdesc[p].clear();
    }
    b.par = 0;
}

void batch_free(Batch &b)
{
    batch_drop(b);
    for (cudaStream_t s : b.pool) cudaStreamDestroy(s);
    for (cudaEvent_t e : b.ev_join) cudaEventDestroy(e);
    if (b.ev_fork) cudaEventDestroy(b.ev_fork);
    b.pool.clear();
    b.ev_join.clear();
    b.ev_fork = nullptr;
}

int batch_step(Ctx &ctx, Batch &B, const std::vector<Case *> &cases, int n)
{
    if (cases.empty() || n <= 0) return MT_OK;
    int rc;
    for (Case *c : cases) {
        if ((rc = amr_prev_sync(ctx, *c))) return rc;
        if ((rc = amr_sync_f(ctx, *c))) return rc;
        if (!c->primed && (rc = prime_fused(ctx, *c))) return rc;
    }
    B.free_stream = ctx.stream;
    if (B.pool.empty()) {
        const int P = 8;
        for (int p = 0; p < P; ++p) {
            cudaStream_t s;
            cudaEvent_t e;
            MT_CUDA(ctx, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            MT_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            B.pool.push_back(s);
            B.ev_join.push_back(e);
        }
        MT_CUDA(ctx, cudaEventCreateWithFlags(&B.ev_fork, cudaEventDisableTiming));
    }
    int Lmax = 0;
    for (Case *c : cases) Lmax = std::max(Lmax, c->d.max_level);
    // capture graph g (0/1: one step from that parity, 2: two steps)
    auto record = [&](int g) -> int {
        const int steps = g == 2 ? 2 : 1;
        BatchRec R;
        R.b = &B;
        R.hdesc = &B.hdesc[g];
        R.hdesc->clear();
        // at most one descriptor per family (3 models x 4 storages) and chunk for every substep
        R.cap = (int64_t)((2 << Lmax) * 12 * steps) *
                (int64_t)((cases.size() + kMaxBatchSlots - 1) / kMaxBatchSlots);
        MT_CUDA(ctx, cudaMallocAsync(&B.ddesc[g], sizeof(BrickBatch) * R.cap, ctx.stream));
        R.dbase = B.ddesc[g];
        for (Case *c : cases) c->no_side = true;
        const int64_t before = ctx.launches;
        cudaGraph_t captured = nullptr;
        cudaError_t e = cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return set_err(ctx, MT_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        int r = MT_OK;
        for (int k = 0; k < steps && !r; ++k) r = record_batch_step(ctx, R, cases);
        e = cudaStreamEndCapture(ctx.stream, &captured);
        for (Case *c : cases) c->no_side = false;
        if (r || e != cudaSuccess) {
            if (captured) cudaGraphDestroy(captured);
            batch_drop(B);
            return r ? r : set_err(ctx, MT_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
        }
        B.graph_launches[g] = ctx.launches - before;
        ctx.launches = before;
        e = cudaGraphInstantiate(&B.graph[g], captured, 0);
        cudaGraphDestroy(captured);
        if (e != cudaSuccess) {
            B.graph[g] = nullptr;
            return set_err(ctx, MT_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        // stream-ordered upload: it lands before the graph's first launch
        MT_CUDA(ctx, cudaMemcpyAsync(B.ddesc[g], R.hdesc->data(), sizeof(BrickBatch) * R.hdesc->size(),
                                     cudaMemcpyHostToDevice, ctx.stream));
        // recording swapped the members' buffers as executing does; undo it
        // so that the caller applies one consistent host-side update per launch
        for (int k = 0; k < steps; ++k)
            for (Case *c : cases) swap_buffers(*c, 0);
        return MT_OK;
    };
    int s = 0;
    while (s < n) {
        const int g = (n - s >= 2) ? 2 : B.par;
        if (!B.graph[g] && (rc = record(g))) return rc;
        MT_CUDA(ctx, cudaGraphLaunch(B.graph[g], ctx.stream));
        ctx.launches += B.graph_launches[g];
        const int steps = g == 2 ? 2 : 1;
        for (int k = 0; k < steps; ++k) {
            for (Case *c : cases) swap_buffers(*c, 0);
            B.par ^= 1;
        }
        s += steps;
        for (Case *c : cases)
            for (int l = 0; l <= c->d.max_level; ++l) c->f_stale |= c->lv[l].bricks;
    }
    return MT_OK;
}

int amr_guard(Ctx &ctx, Case &c, int *flags)
{
    if (int rc = amr_sync_f(ctx, c)) return rc;
    MT_CUDA(ctx, cudaMemsetAsync(c.dev_err, 0, sizeof(int), ctx.stream));
    int rc = amr_dispatch(c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return AmrOps<S>::guard(ctx, c);
    });
    if (rc) return rc;
    MT_CUDA(ctx, cudaMemcpyAsync(flags, c.dev_err, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    return MT_OK;
}

// FP64 per-level and volume-weighted sums of mass, momentum and kinetic
// energy (host out[(max_level + 2) * 5]); the streamed f is rebuilt first
// where the fused schedule does not store it
int amr_reduce(Ctx &ctx, Case &c, double *h_out)
{
    if (int rc = amr_sync_f(ctx, c)) return rc;
    const size_t nb = sizeof(double) * 5 * (size_t)(c.d.max_level + 2);
    double *d = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&d, nb, ctx.stream));
    int rc = amr_dispatch(c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return AmrOps<S>::reduce(ctx, c, d);
    });
    if (!rc) MT_CUDA(ctx, cudaMemcpyAsync(h_out, d, nb, cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    cudaFreeAsync(d, ctx.stream);
    return rc;
}

// LBM_Manager::infoPrint's per-level diagnostics (mt_case_info): the
// end-of-step macros are current after every coarse step under both
// schedules, so no population sync is needed
int amr_info(Ctx &ctx, Case &c, double *h_out)
{
    const size_t nb = sizeof(double) * 4 * (size_t)(c.d.max_level + 1);
    double *d = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&d, nb, ctx.stream));
    int rc = amr_dispatch(c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return AmrOps<S>::info(ctx, c, d);
    });
    if (!rc) MT_CUDA(ctx, cudaMemcpyAsync(h_out, d, nb, cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    cudaFreeAsync(d, ctx.stream);
    return rc;
}

// populations of one level as FP64 [Q][n] (host buffers), in either direction
int amr_get(Ctx &ctx, Case &c, int level, double *h_f, double *h_fcol)
{
    if (int rc = amr_sync_f(ctx, c)) return rc;
    Level &lv = c.lv[level];
    if (!lv.n) return MT_OK;
    const size_t nb = sizeof(double) * (size_t)c.d.q * (size_t)lv.n;
    double *d = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&d, nb, ctx.stream));
    int rc = MT_OK;
    for (int which = 0; which < 2 && !rc; ++which) {
        double *dst = which == 0 ? h_f : h_fcol;
        if (!dst) continue;
        rc = amr_dispatch(c, [&](auto *tag) {
            using S = std::remove_pointer_t<decltype(tag)>;
            return AmrOps<S>::get(ctx, c, level, which, d);
        });
        if (!rc) MT_CUDA(ctx, cudaMemcpyAsync(dst, d, nb, cudaMemcpyDeviceToHost, ctx.stream));
        MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    }
    cudaFreeAsync(d, ctx.stream);
    return rc;
}

int amr_set(Ctx &ctx, Case &c, int level, const double *h_f, const double *h_fcol)
{
    if (int rc = amr_sync_f(ctx, c)) return rc;
    c.prev_stale = true;
    Level &lv = c.lv[level];
    if (!lv.n) return MT_OK;
    const size_t nb = sizeof(double) * (size_t)c.d.q * (size_t)lv.n;
    double *d = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&d, nb, ctx.stream));
    int rc = MT_OK;
    for (int which = 0; which < 2 && !rc; ++which) {
        const double *src = which == 0 ? h_f : h_fcol;
        if (!src) continue;
        MT_CUDA(ctx, cudaMemcpyAsync(d, src, nb, cudaMemcpyHostToDevice, ctx.stream));
        rc = amr_dispatch(c, [&](auto *tag) {
            using S = std::remove_pointer_t<decltype(tag)>;
            return AmrOps<S>::set(ctx, c, level, which, d);
        });
    }
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    cudaFreeAsync(d, ctx.stream);
    return rc;
}

int amr_macros(Ctx &ctx, Case &c, int level, double *h_rho, double *h_u)
{
    Level &lv = c.lv[level];
    if (!lv.n) return MT_OK;
    double *d = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&d, sizeof(double) * 4 * lv.n, ctx.stream));
    int rc = amr_dispatch(c, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return AmrOps<S>::macros_out(ctx, c, level, d, d + lv.n);
    });
    if (!rc) {
        if (h_rho) MT_CUDA(ctx, cudaMemcpyAsync(h_rho, d, sizeof(double) * lv.n, cudaMemcpyDeviceToHost, ctx.stream));
        if (h_u) MT_CUDA(ctx, cudaMemcpyAsync(h_u, d + lv.n, sizeof(double) * 3 * lv.n, cudaMemcpyDeviceToHost, ctx.stream));
    }
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    cudaFreeAsync(d, ctx.stream);
    return rc;
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
