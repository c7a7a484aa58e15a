// Lattice classification on the device: the per-level index sets of
// Lat_Manager (Lat_Manager.hpp:245-316) for nested refinement boxes and an
// analytic sphere or a triangulated surface, generated directly as raw
// (key, set) pairs for the build (mt_case_generate).  It restates, set for
// set, what the host mesher (mortontrie_amr_b200/mesh.py) produces --
// boundary shell split into the 26 lat_bc sets, F2C = 1-cell shell of each
// refinement box, C2F = 2-cell shell of each refined level, ghost layers
// from Q-neighbours, the voxelised solid with its wall distances
// (Lat_Voxelize.cpp:1252-1285 semantics) or the direct-forcing band -- and
// raises the same contract errors.  Compiled without FMA contraction so the
// wall distances equal the host's.  amr_remap (mt_case_remap) dispatches the
// state remap onto such a lattice.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "mt_internal.hpp"

namespace mt {

namespace {

// payload byte 0: the build's set code (0 lat_f, 1 F2C, 2 C2F, 5 solid,
// 16 + b lat_bc[b]); bit 8: in the forcing band; 0xff: not stored
enum : uint32_t { P_LATF = 0, P_F2C = 1, P_C2F = 2, P_SF = 5, P_NONE = 0xffu, P_BAND = 0x100u };
enum : int { MERR_BOX_BC = 1, MERR_BOX_C2F = 2, MERR_GHOST = 4, MERR_SOLID = 8, MERR_BAND = 16 };

struct Box {
    int64_t lo[3], hi[3];
    MT_HD int64_t n() const { return (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]); }
};

// a set of cells of one level as a dense mask over a box (mt_case_set_region)
struct RegionMask {
    const uint8_t *m;
    int64_t lo[3], n[3];
    MT_HD bool has(int64_t x, int64_t y, int64_t z) const
    {
        const int64_t a = x - lo[0], b = y - lo[1], c = z - lo[2];
        if (a < 0 || b < 0 || c < 0 || a >= n[0] || b >= n[1] || c >= n[2]) return false;
        return m[(a * n[1] + b) * n[2] + c] != 0;
    }
    // in the set with one of its 26 neighbours outside it
    MT_HD bool edge(int64_t x, int64_t y, int64_t z) const
    {
        if (!has(x, y, z)) return false;
        for (int d = 0; d < 27; ++d)
            if (d != 13 && !has(x + d % 3 - 1, y + (d / 3) % 3 - 1, z + d / 9 - 1)) return true;
        return false;
    }
};

struct LevelGen {
    int level, L, q;
    int64_t ext[3];  // level extent in its own cells
    int bc[3];       // boundary shell on this axis (level 0)
    int per[3];      // periodic axis
    Box dom;         // cells of this level (for a region: the box of its children)
    int dom_region;  // the level's cells are the children of dreg's cells
    RegionMask dreg; // in level-(l-1) cells
    int has_ref;     // refinement box of this level present
    Box ref;         // in this level's cells
    int ref_region;  // the refined cells are rreg's (instead of the box ref)
    RegionMask rreg; // in this level's cells
    int sphere;      // 0 none, 1 solid + links, 2 band, 3 triangulated surface (finest level only)
    double cx, cy, cz, r, amp, slack;  // finest-level units
    int8_t side_bc[27];                // lat_bc index of a (-1, 0, 1)^3 side combination
    // surface: crossings of the +x centre lines with the triangles, per
    // finest (y, z) column over the finest box (CSR)
    const int32_t *col_off;
    const double *col_x;
    int64_t col_lo[2], col_n[2];
};

MT_HD uint64_t level_key(int L, int l, int64_t x, int64_t y, int64_t z)
{
    const int sh = L - l;
    return dilate3((uint64_t)x << sh) | (dilate3((uint64_t)y << sh) << 1) | (dilate3((uint64_t)z << sh) << 2);
}

// every cell of the level's box: its key (~0 when not stored) and payload
__global__ void k_classify(LevelGen g, uint64_t *key, uint32_t *pay, int *err)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nx = g.dom.hi[0] - g.dom.lo[0], ny = g.dom.hi[1] - g.dom.lo[1];
    if (t >= g.dom.n()) return;
    const int64_t x = g.dom.lo[0] + t % nx, y = g.dom.lo[1] + (t / nx) % ny, z = g.dom.lo[2] + t / (nx * ny);
    const int64_t c[3] = {x, y, z};
    if (g.dom_region && !g.dreg.has(x >> 1, y >> 1, z >> 1)) {
        // inside the box of the region's children but not one of them
        if (g.ref_region && g.rreg.has(x, y, z)) atomicOr(err, MERR_BOX_C2F);
        key[t] = ~0ull;
        pay[t] = P_NONE;
        return;
    }
    int bcb = -1;
    if (g.level == 0) {
        int side[3] = {0, 0, 0};
        for (int a = 0; a < 3; ++a)
            if (g.bc[a]) side[a] = c[a] == 0 ? -1 : (c[a] == g.ext[a] - 1 ? 1 : 0);
        if (side[0] || side[1] || side[2]) bcb = g.side_bc[(side[0] + 1) + 3 * (side[1] + 1) + 9 * (side[2] + 1)];
    }
    bool f2c = false, removed = false;
    if (g.has_ref) {
        bool inside = true, shell = false;
        if (g.ref_region) {
            inside = g.rreg.has(x, y, z);
            shell = inside && g.rreg.edge(x, y, z);
        } else {
            for (int a = 0; a < 3; ++a) {
                inside &= c[a] >= g.ref.lo[a] && c[a] < g.ref.hi[a];
                shell |= c[a] < g.ref.lo[a] + 1 || c[a] >= g.ref.hi[a] - 1;
            }
        }
        f2c = inside && shell;
        removed = inside && !shell;
        if (inside && bcb >= 0) atomicOr(err, MERR_BOX_BC);
    }
    bool c2f = false;
    if (g.dom_region)
        c2f = g.dreg.edge(x >> 1, y >> 1, z >> 1);  // a child of a coarser F2C cell
    else if (g.level > 0)
        for (int a = 0; a < 3; ++a) c2f |= c[a] < g.dom.lo[a] + 2 || c[a] >= g.dom.hi[a] - 2;
    if (c2f && f2c) atomicOr(err, MERR_BOX_C2F);
    uint32_t p;
    if (removed)
        p = P_NONE;
    else if (bcb >= 0)
        p = 16u + (uint32_t)bcb;
    else if (f2c)
        p = P_F2C;
    else if (c2f)
        p = P_C2F;
    else
        p = P_LATF;
    if (p == P_LATF && g.sphere && g.level == g.L) {
        const double px = (double)x + 0.5 - g.cx, py = (double)y + 0.5 - g.cy, pz = (double)z + 0.5 - g.cz;
        if (g.sphere == 1) {
            if (px * px + py * py + pz * pz < g.r * g.r) p = P_SF;
        } else if (g.sphere == 3) {
            const int64_t cy = y - g.col_lo[0], cz = z - g.col_lo[1];
            if (cy >= 0 && cy < g.col_n[0] && cz >= 0 && cz < g.col_n[1]) {
                const int64_t col = cy * g.col_n[1] + cz;
                const double xc = (double)x + 0.5;
                int above = 0;
                for (int32_t k = g.col_off[col]; k < g.col_off[col + 1]; ++k) above += g.col_x[k] > xc;
                if (above & 1) p = P_SF;
            }
        } else {
            const double qy = fmin(fmax(py, -g.amp), g.amp);
            const double dmin = sqrt(px * px + (py - qy) * (py - qy) + pz * pz);
            const double ay = fabs(py) + g.amp;
            const double dmax = sqrt(px * px + ay * ay + pz * pz);
            if ((dmin <= g.r + 2.7) && (dmax >= g.r - 2.7 - g.slack)) p |= P_BAND;
        }
    }
    key[t] = p == P_NONE ? ~0ull : level_key(g.L, g.level, x, y, z);
    pay[t] = p;
}

// flags of the payloads: mode 0 set code == v, 1 band bit
__global__ void k_flags(const uint32_t *pay, int64_t n, int mode, uint32_t v, uint8_t *flag)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    flag[t] = mode == 0 ? ((pay[t] & 0xffu) == v) : ((pay[t] & P_BAND) != 0);
}

// neighbour keys (Q - 1 per source cell), periodic axes wrapped; ~0 when a
// coordinate falls below zero (the host mesher's filter)
template <int Q>
__global__ void k_nbr_keys(const uint64_t *src, int64_t ns, LevelGen g, uint64_t *out)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= ns * (Q - 1)) return;
    const int64_t j = t / (Q - 1);
    const int k = (int)(t - j * (Q - 1)) + 1;
    const uint64_t key = src[j];
    const int sh = g.L - g.level;
    int64_t c[3] = {(int64_t)(compact3(key) >> sh), (int64_t)(compact3(key >> 1) >> sh),
                    (int64_t)(compact3(key >> 2) >> sh)};
    const int e[3] = {ex(k), ey(k), ez(k)};
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
        int64_t v = c[a] + e[a];
        if (g.per[a]) v = ((v % g.ext[a]) + g.ext[a]) % g.ext[a];
        if (v < 0) ok = false;
        c[a] = v;
    }
    out[t] = ok ? level_key(g.L, g.level, c[0], c[1], c[2]) : ~0ull;
}

// flag[t]: key valid and (mode 0) in neither a nor b, (mode 1) in a
__global__ void k_member(const uint64_t *keys, int64_t n, const uint64_t *a, int64_t na, const uint64_t *b,
                         int64_t nb, int mode, uint8_t *flag)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint64_t k = keys[t];
    bool f = false;
    if (k != ~0ull) {
        const bool ia = na && find_key(a, na, k) >= 0;
        const bool ib = nb && find_key(b, nb, k) >= 0;
        f = mode == 0 ? (!ia && !ib) : ia;
    }
    flag[t] = f;
}

__global__ void k_check_in(const uint64_t *keys, int64_t n, const uint64_t *a, int64_t na, const uint64_t *b,
                           int64_t nb, int flag, int *err)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint64_t k = keys[t];
    if (k == ~0ull) return;
    if ((na && find_key(a, na, k) >= 0) || (nb && find_key(b, nb, k) >= 0)) atomicOr(err, flag);
}

// wall distances of the finest fluid cells (mesh.py _sphere_links, same
// operation order); hit[j] = 1 when some link crosses the sphere
template <int Q>
__global__ void k_links(const uint64_t *keys, int64_t n, double cx, double cy, double cz, double r, double *rows,
                        uint8_t *hit)
{
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint64_t key = keys[j];
    const double px = (double)(int64_t)compact3(key) + 0.5 - cx;
    const double py = (double)(int64_t)compact3(key >> 1) + 0.5 - cy;
    const double pz = (double)(int64_t)compact3(key >> 2) + 0.5 - cz;
    const double c0 = px * px + py * py + pz * pz - r * r;
    bool any = false;
    for (int d = 1; d < Q; ++d) {
        const double a = (double)(ex(d) * ex(d) + ey(d) * ey(d) + ez(d) * ez(d));
        const double b = 2.0 * (px * ex(d) + py * ey(d) + pz * ez(d));
        const double disc = b * b - 4.0 * a * c0;
        double t = -1.0;
        if (disc >= 0.0) {
            const double tt = (-b - sqrt(disc)) / (2.0 * a);
            if (tt >= 0.0 && tt <= 1.0) t = tt;
        }
        rows[j * (Q - 1) + (d - 1)] = t;
        any |= t != -1.0;
    }
    hit[j] = any ? 1 : 0;
}

__global__ void k_gather_rows(const int64_t *idx, int64_t nd, const double *rows, const uint64_t *keys, int w,
                              double *out, uint64_t *okey)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= nd * w) return;
    const int64_t j = t / w;
    out[t] = rows[idx[j] * w + (t - j * w)];
    if (t - j * w == 0) okey[j] = keys[idx[j]];
}

__global__ void k_codes(const uint32_t *pay, int64_t n, uint8_t *code)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) code[t] = (uint8_t)(pay[t] & 0xffu);
}

__global__ void k_fill_u8(uint8_t *p, int64_t n, uint8_t v)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t < n) p[t] = v;
}

// ---- triangulated surfaces (mesh.py column_crossings / link_hits, same
// operation order) -------------------------------------------------------
struct Tri {
    double v[3][3];
};

MT_HD double edge_orient(double uy, double uz, double vy, double vz, double py, double pz)
{
    const bool swap = (uy > vy) || (uy == vy && uz > vz);
    const double Py = swap ? vy : uy, Pz = swap ? vz : uz, Ry = swap ? uy : vy, Rz = swap ? uz : vz;
    const double o = (Ry - Py) * (pz - Pz) - (Rz - Pz) * (py - Py);
    return swap ? -o : o;
}

// crossing of the line {(t, py, pz)} with the triangle: x, or false
MT_HD bool column_crossing(const Tri &t, double py, double pz, double *x)
{
    const double *a = t.v[0], *b = t.v[1], *c = t.v[2];
    const double area = (b[1] - a[1]) * (c[2] - a[2]) - (b[2] - a[2]) * (c[1] - a[1]);
    if (area == 0.0) return false;
    const double *vs[3] = {a, area > 0.0 ? b : c, area > 0.0 ? c : b};
    for (int i = 0; i < 3; ++i) {
        const double *u = vs[i], *v = vs[(i + 1) % 3];
        const double o = edge_orient(u[1], u[2], v[1], v[2], py, pz);
        const double dy = v[1] - u[1], dz = v[2] - u[2];
        const bool top_left = (dz < 0.0) || (dz == 0.0 && dy < 0.0);
        if (!(o > 0.0 || (o == 0.0 && top_left))) return false;
    }
    const double ny = (b[2] - a[2]) * (c[0] - a[0]) - (b[0] - a[0]) * (c[2] - a[2]);
    const double nz = (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0]);
    *x = a[0] - (ny * (py - a[1]) + nz * (pz - a[2])) / area;
    return true;
}

struct ColRange {
    int64_t y0, y1, z0, z1;  // inclusive, clipped to the columns
};
MT_HD ColRange tri_columns(const Tri &t, const int64_t lo[2], const int64_t n[2])
{
    double ylo = fmin(fmin(t.v[0][1], t.v[1][1]), t.v[2][1]), yhi = fmax(fmax(t.v[0][1], t.v[1][1]), t.v[2][1]);
    double zlo = fmin(fmin(t.v[0][2], t.v[1][2]), t.v[2][2]), zhi = fmax(fmax(t.v[0][2], t.v[1][2]), t.v[2][2]);
    ColRange r;
    r.y0 = (int64_t)ceil(ylo - 0.5);
    r.y1 = (int64_t)floor(yhi - 0.5);
    r.z0 = (int64_t)ceil(zlo - 0.5);
    r.z1 = (int64_t)floor(zhi - 0.5);
    r.y0 = r.y0 > lo[0] ? r.y0 : lo[0];
    r.z0 = r.z0 > lo[1] ? r.z0 : lo[1];
    r.y1 = r.y1 < lo[0] + n[0] - 1 ? r.y1 : lo[0] + n[0] - 1;
    r.z1 = r.z1 < lo[1] + n[1] - 1 ? r.z1 : lo[1] + n[1] - 1;
    return r;
}

// pass 0: count the crossings per column; pass 1: write their x
__global__ void k_tri_columns(const Tri *tri, int64_t ntri, LevelGen g, int pass, int32_t *cnt, int32_t *cursor,
                              double *col_x)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= ntri) return;
    const Tri t = tri[i];
    const ColRange r = tri_columns(t, g.col_lo, g.col_n);
    for (int64_t y = r.y0; y <= r.y1; ++y)
        for (int64_t z = r.z0; z <= r.z1; ++z) {
            double x;
            if (!column_crossing(t, (double)y + 0.5, (double)z + 0.5, &x)) continue;
            const int64_t col = (y - g.col_lo[0]) * g.col_n[1] + (z - g.col_lo[1]);
            if (pass == 0)
                atomicAdd(&cnt[col], 1);
            else
                col_x[atomicAdd(&cursor[col], 1)] = x;
        }
}

struct BinBox {
    int64_t lo[3], n[3];
};
// finest cells whose links can reach the triangle: [ceil(lo - 1.5), floor(hi + 0.5)] per axis, clipped
MT_HD void tri_bins(const Tri &t, const BinBox &b, int64_t r0[3], int64_t r1[3])
{
    for (int a = 0; a < 3; ++a) {
        const double lo = fmin(fmin(t.v[0][a], t.v[1][a]), t.v[2][a]);
        const double hi = fmax(fmax(t.v[0][a], t.v[1][a]), t.v[2][a]);
        int64_t u0 = (int64_t)ceil(lo - 1.5), u1 = (int64_t)floor(hi + 0.5);
        r0[a] = u0 > b.lo[a] ? u0 : b.lo[a];
        r1[a] = u1 < b.lo[a] + b.n[a] - 1 ? u1 : b.lo[a] + b.n[a] - 1;
    }
}

__global__ void k_tri_bins(const Tri *tri, int64_t ntri, BinBox b, int pass, int32_t *cnt, int32_t *cursor,
                           int32_t *bin_tri)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= ntri) return;
    int64_t r0[3], r1[3];
    tri_bins(tri[i], b, r0, r1);
    for (int64_t x = r0[0]; x <= r1[0]; ++x)
        for (int64_t y = r0[1]; y <= r1[1]; ++y)
            for (int64_t z = r0[2]; z <= r1[2]; ++z) {
                const int64_t cell = ((x - b.lo[0]) * b.n[1] + (y - b.lo[1])) * b.n[2] + (z - b.lo[2]);
                if (pass == 0)
                    atomicAdd(&cnt[cell], 1);
                else
                    bin_tri[atomicAdd(&cursor[cell], 1)] = (int32_t)i;
            }
}

constexpr double kLinkEps = 1e-10;

// wall distances of the finest fluid cells against the surface's triangles
// (smallest normalised distance per link); hit[j] = 1 when any link crosses
template <int Q>
__global__ void k_links_surface(const uint64_t *keys, int64_t n, const Tri *tri, BinBox b, const int32_t *bin_off,
                                const int32_t *bin_tri, double *rows, uint8_t *hit)
{
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint64_t key = keys[j];
    const int64_t c[3] = {(int64_t)compact3(key), (int64_t)compact3(key >> 1), (int64_t)compact3(key >> 2)};
    double best[Q - 1];
    for (int k = 0; k < Q - 1; ++k) best[k] = -1.0;
    bool inbox = true;
    for (int a = 0; a < 3; ++a) inbox &= c[a] >= b.lo[a] && c[a] < b.lo[a] + b.n[a];
    if (inbox) {
        const int64_t cell = ((c[0] - b.lo[0]) * b.n[1] + (c[1] - b.lo[1])) * b.n[2] + (c[2] - b.lo[2]);
        const double px = (double)c[0] + 0.5, py = (double)c[1] + 0.5, pz = (double)c[2] + 0.5;
        for (int32_t e = bin_off[cell]; e < bin_off[cell + 1]; ++e) {
            const Tri t = tri[bin_tri[e]];
            const double *v1 = t.v[0], *v2 = t.v[1], *v3 = t.v[2];
            const double e1[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
            const double e2[3] = {v3[0] - v1[0], v3[1] - v1[1], v3[2] - v1[2]};
            const double sx = px - v1[0], sy = py - v1[1], sz = pz - v1[2];
            for (int k = 1; k < Q; ++k) {
                const double gx = (double)ex(k), gy = (double)ey(k), gz = (double)ez(k);
                const double mag = sqrt(gx * gx + gy * gy + gz * gz);
                const double dx = gx / mag, dy = gy / mag, dz = gz / mag;
                const double s1[3] = {dy * e2[2] - dz * e2[1], dz * e2[0] - dx * e2[2], dx * e2[1] - dy * e2[0]};
                const double s2[3] = {sy * e1[2] - sz * e1[1], sz * e1[0] - sx * e1[2], sx * e1[1] - sy * e1[0]};
                const double s1e1 = s1[0] * e1[0] + s1[1] * e1[1] + s1[2] * e1[2];
                if (s1e1 == 0.0) continue;
                const double tt = (s2[0] * e2[0] + s2[1] * e2[1] + s2[2] * e2[2]) / s1e1;
                const double b1 = (s1[0] * sx + s1[1] * sy + s1[2] * sz) / s1e1;
                const double b2 = (s2[0] * dx + s2[1] * dy + s2[2] * dz) / s1e1;
                const double b0 = 1.0 - b1 - b2;
                if (!(tt >= kLinkEps && b1 >= -kLinkEps && b2 >= -kLinkEps && b0 >= -kLinkEps)) continue;
                const double ix = b0 * v1[0] + b1 * v2[0] + b2 * v3[0];
                const double iy = b0 * v1[1] + b1 * v2[1] + b2 * v3[1];
                const double iz = b0 * v1[2] + b1 * v2[2] + b2 * v3[2];
                const double dist = sqrt((ix - px) * (ix - px) + (iy - py) * (iy - py) + (iz - pz) * (iz - pz));
                const double nrm = dist / mag;
                if (!(nrm >= 0.0 && nrm <= 1.0)) continue;
                if (best[k - 1] == -1.0 || nrm < best[k - 1]) best[k - 1] = nrm;
            }
        }
    }
    bool any = false;
    for (int k = 0; k < Q - 1; ++k) {
        rows[j * (Q - 1) + k] = best[k];
        any |= best[k] != -1.0;
    }
    hit[j] = any ? 1 : 0;
}

// device buffer with stream-ordered allocation and release
template <class T> struct DBuf {
    T *p = nullptr;
    int64_t n = 0;
    cudaStream_t s = nullptr;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    int alloc(Ctx &ctx, int64_t count)
    {
        if (p) cudaFreeAsync(p, s);
        s = ctx.stream;
        n = count;
        MT_CUDA(ctx, cudaMallocAsync(&p, sizeof(T) * std::max<int64_t>(count, 1), s));
        return MT_OK;
    }
    ~DBuf()
    {
        if (p) cudaFreeAsync(p, s);
    }
    T *release()
    {
        T *q = p;
        p = nullptr;
        return q;
    }
};

// keys[flag] in order -> out (count on the host)
int select_flagged(Ctx &ctx, const uint64_t *keys, const uint8_t *flag, int64_t n, DBuf<uint64_t> &out)
{
    if (int rc = out.alloc(ctx, n)) return rc;
    if (!n) {
        out.n = 0;
        return MT_OK;
    }
    DBuf<int> cnt;
    if (int rc = cnt.alloc(ctx, 1)) return rc;
    size_t tb = 0;
    MT_CUDA(ctx, cub::DeviceSelect::Flagged(nullptr, tb, keys, flag, out.p, cnt.p, (int)n, ctx.stream));
    DBuf<char> tmp;
    if (int rc = tmp.alloc(ctx, (int64_t)tb)) return rc;
    MT_CUDA(ctx, cub::DeviceSelect::Flagged(tmp.p, tb, keys, flag, out.p, cnt.p, (int)n, ctx.stream));
    int h = 0;
    MT_CUDA(ctx, cudaMemcpyAsync(&h, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    out.n = h;
    return MT_OK;
}

// sorted unique keys of an unsorted array (sentinels sort last and are kept once)
int sort_unique(Ctx &ctx, const uint64_t *keys, int64_t n, DBuf<uint64_t> &out)
{
    if (int rc = out.alloc(ctx, n)) return rc;
    if (!n) {
        out.n = 0;
        return MT_OK;
    }
    DBuf<uint64_t> sorted;
    if (int rc = sorted.alloc(ctx, n)) return rc;
    DBuf<int> cnt;
    if (int rc = cnt.alloc(ctx, 1)) return rc;
    size_t t1 = 0, t2 = 0;
    MT_CUDA(ctx, cub::DeviceRadixSort::SortKeys(nullptr, t1, keys, sorted.p, (int)n, 0, 64, ctx.stream));
    MT_CUDA(ctx, cub::DeviceSelect::Unique(nullptr, t2, sorted.p, out.p, cnt.p, (int)n, ctx.stream));
    DBuf<char> tmp;
    if (int rc = tmp.alloc(ctx, (int64_t)std::max(t1, t2))) return rc;
    MT_CUDA(ctx, cub::DeviceRadixSort::SortKeys(tmp.p, t1, keys, sorted.p, (int)n, 0, 64, ctx.stream));
    MT_CUDA(ctx, cub::DeviceSelect::Unique(tmp.p, t2, sorted.p, out.p, cnt.p, (int)n, ctx.stream));
    int h = 0;
    MT_CUDA(ctx, cudaMemcpyAsync(&h, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    out.n = h;
    return MT_OK;
}

int nbr_keys(Ctx &ctx, const LevelGen &g, const uint64_t *src, int64_t ns, DBuf<uint64_t> &out)
{
    const int64_t m = ns * (g.q - 1);
    if (int rc = out.alloc(ctx, m)) return rc;
    if (!m) return MT_OK;
    if (g.q == 19)
        k_nbr_keys<19><<<grid_for(m, 256), 256, 0, ctx.stream>>>(src, ns, g, out.p);
    else
        k_nbr_keys<27><<<grid_for(m, 256), 256, 0, ctx.stream>>>(src, ns, g, out.p);
    MT_LAUNCHED(ctx);
    return MT_OK;
}

// the sorted keys of one set code among the level's sorted stored cells
int set_keys(Ctx &ctx, const uint64_t *skey, const uint32_t *spay, int64_t ns, int mode, uint32_t v,
             DBuf<uint64_t> &out)
{
    DBuf<uint8_t> flag;
    if (int rc = flag.alloc(ctx, ns)) return rc;
    if (ns) {
        k_flags<<<grid_for(ns, 256), 256, 0, ctx.stream>>>(spay, ns, mode, v, flag.p);
        MT_LAUNCHED(ctx);
    }
    return select_flagged(ctx, skey, flag.p, ns, out);
}

// the surface's tables on the device: triangles in finest-cell units, the
// column crossings (CSR over the finest box's (y, z) columns) and the link
// bins (CSR of triangle indices per finest cell of the bin box)
struct SurfaceTables {
    DBuf<Tri> tri;
    DBuf<int32_t> col_off, bin_off, bin_tri;
    DBuf<double> col_x;
    int64_t col_lo[2] = {0, 0}, col_n[2] = {0, 0};
    BinBox box{};
};

int csr_offsets(Ctx &ctx, DBuf<int32_t> &cnt, int64_t n, DBuf<int32_t> &off, int64_t *total)
{
    if (int rc = off.alloc(ctx, n + 1)) return rc;
    size_t tb = 0;
    MT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.p, off.p, (int)(n + 1), ctx.stream));
    DBuf<char> tmp;
    if (int rc = tmp.alloc(ctx, (int64_t)tb)) return rc;
    MT_CUDA(ctx, cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.p, off.p, (int)(n + 1), ctx.stream));
    int32_t h = 0;
    MT_CUDA(ctx, cudaMemcpyAsync(&h, off.p + n, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    *total = h;
    return MT_OK;
}

int surface_tables(Ctx &ctx, const std::vector<double> &h_tri, int L, const Box &fdom, SurfaceTables &st)
{
    const int64_t nt = (int64_t)h_tri.size() / 9;
    std::vector<Tri> tris((size_t)nt);
    const double sc = (double)(1 << L);
    for (int64_t i = 0; i < nt; ++i)
        for (int v = 0; v < 3; ++v)
            for (int a = 0; a < 3; ++a) tris[(size_t)i].v[v][a] = h_tri[(size_t)(9 * i + 3 * v + a)] * sc;
    if (int rc = st.tri.alloc(ctx, nt)) return rc;
    MT_CUDA(ctx, cudaMemcpyAsync(st.tri.p, tris.data(), sizeof(Tri) * nt, cudaMemcpyHostToDevice, ctx.stream));
    // columns of the finest box; entries bounded on the host before the int32 offsets
    st.col_lo[0] = fdom.lo[1];
    st.col_lo[1] = fdom.lo[2];
    st.col_n[0] = std::max<int64_t>(0, fdom.hi[1] - fdom.lo[1]);
    st.col_n[1] = std::max<int64_t>(0, fdom.hi[2] - fdom.lo[2]);
    int64_t col_bound = 0, bin_bound = 0;
    int64_t blo[3] = {INT64_MAX, INT64_MAX, INT64_MAX}, bhi[3] = {INT64_MIN, INT64_MIN, INT64_MIN};
    for (const Tri &t : tris) {
        const ColRange r = tri_columns(t, st.col_lo, st.col_n);
        if (r.y1 >= r.y0 && r.z1 >= r.z0) col_bound += (r.y1 - r.y0 + 1) * (r.z1 - r.z0 + 1);
        for (int a = 0; a < 3; ++a) {
            const double lo = std::fmin(std::fmin(t.v[0][a], t.v[1][a]), t.v[2][a]);
            const double hi = std::fmax(std::fmax(t.v[0][a], t.v[1][a]), t.v[2][a]);
            blo[a] = std::min<int64_t>(blo[a], (int64_t)std::ceil(lo - 1.5));
            bhi[a] = std::max<int64_t>(bhi[a], (int64_t)std::floor(hi + 0.5));
        }
    }
    bool empty = nt == 0;
    for (int a = 0; a < 3; ++a) {
        blo[a] = std::max(blo[a], fdom.lo[a]);
        bhi[a] = std::min(bhi[a], fdom.hi[a] - 1);
        empty |= bhi[a] < blo[a];
    }
    for (int a = 0; a < 3; ++a) {
        st.box.lo[a] = empty ? 0 : blo[a];
        st.box.n[a] = empty ? 0 : bhi[a] - blo[a] + 1;
    }
    if (!empty)
        for (const Tri &t : tris) {
            int64_t r0[3], r1[3];
            tri_bins(t, st.box, r0, r1);
            int64_t v = 1;
            for (int a = 0; a < 3; ++a) v *= std::max<int64_t>(0, r1[a] - r0[a] + 1);
            bin_bound += v;
        }
    const int64_t ncol = st.col_n[0] * st.col_n[1];
    const int64_t nbin = st.box.n[0] * st.box.n[1] * st.box.n[2];
    if (col_bound > INT32_MAX || bin_bound > INT32_MAX || ncol > INT32_MAX - 1 || nbin > INT32_MAX - 1)
        return set_err(ctx, MT_ERR_ARG, "surface too large for the crossing and link tables");
    LevelGen g{};
    g.col_lo[0] = st.col_lo[0];
    g.col_lo[1] = st.col_lo[1];
    g.col_n[0] = st.col_n[0];
    g.col_n[1] = st.col_n[1];
    {
        DBuf<int32_t> cnt, cur;
        if (int rc = cnt.alloc(ctx, ncol + 1)) return rc;
        MT_CUDA(ctx, cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (ncol + 1), ctx.stream));
        if (nt && ncol) {
            k_tri_columns<<<grid_for(nt, 128), 128, 0, ctx.stream>>>(st.tri.p, nt, g, 0, cnt.p, nullptr, nullptr);
            MT_LAUNCHED(ctx);
        }
        int64_t total = 0;
        if (int rc = csr_offsets(ctx, cnt, ncol, st.col_off, &total)) return rc;
        if (int rc = st.col_x.alloc(ctx, total)) return rc;
        if (int rc = cur.alloc(ctx, ncol + 1)) return rc;
        MT_CUDA(ctx, cudaMemcpyAsync(cur.p, st.col_off.p, sizeof(int32_t) * (ncol + 1), cudaMemcpyDeviceToDevice,
                                     ctx.stream));
        if (total) {
            k_tri_columns<<<grid_for(nt, 128), 128, 0, ctx.stream>>>(st.tri.p, nt, g, 1, nullptr, cur.p, st.col_x.p);
            MT_LAUNCHED(ctx);
        }
    }
    {
        DBuf<int32_t> cnt, cur;
        if (int rc = cnt.alloc(ctx, nbin + 1)) return rc;
        MT_CUDA(ctx, cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (nbin + 1), ctx.stream));
        if (nt && nbin) {
            k_tri_bins<<<grid_for(nt, 128), 128, 0, ctx.stream>>>(st.tri.p, nt, st.box, 0, cnt.p, nullptr, nullptr);
            MT_LAUNCHED(ctx);
        }
        int64_t total = 0;
        if (int rc = csr_offsets(ctx, cnt, nbin, st.bin_off, &total)) return rc;
        if (int rc = st.bin_tri.alloc(ctx, total)) return rc;
        if (int rc = cur.alloc(ctx, nbin + 1)) return rc;
        MT_CUDA(ctx, cudaMemcpyAsync(cur.p, st.bin_off.p, sizeof(int32_t) * (nbin + 1), cudaMemcpyDeviceToDevice,
                                     ctx.stream));
        if (total) {
            k_tri_bins<<<grid_for(nt, 128), 128, 0, ctx.stream>>>(st.tri.p, nt, st.box, 1, nullptr, cur.p,
                                                                 st.bin_tri.p);
            MT_LAUNCHED(ctx);
        }
    }
    return MT_OK;
}

}  // namespace

// the state of case src carried onto case dst (another lattice of the same
// model and storage): AmrOps<S>::remap per level, then dst's direct-forcing
// step counter follows src's.  counts[4 * l + kind] receives the cells of
// each kind.
int amr_remap(Ctx &ctx, Case &dst, Case &src, int64_t *counts)
{
    dst.prev_stale = true;
    if (int rc = amr_sync_f(ctx, src)) return rc;
    if (int rc = amr_sync_f(ctx, dst)) return rc;
    int rc = amr_dispatch(dst, [&](auto *tag) {
        using S = std::remove_pointer_t<decltype(tag)>;
        return AmrOps<S>::remap(ctx, dst, src, counts);
    });
    if (rc) return rc;
    if (dst.tstep && src.tstep)
        MT_CUDA(ctx, cudaMemcpyAsync(dst.tstep, src.tstep, sizeof(long long), cudaMemcpyDeviceToDevice, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    dst.primed = false;
    return MT_OK;
}

// raw sets of every level, the dis table or the band, then the build
int amr_generate(Ctx &ctx, Case &c, const mt_mesh_spec &sp)
{
    const int L = c.d.max_level;
    const int q = c.d.q;
    static const int8_t sides[26][3] = {
        {-1, 0, 0}, {1, 0, 0},   {0, -1, 0},  {0, 1, 0},   {0, 0, -1},  {0, 0, 1},   {1, 1, 0},
        {-1, 1, 0}, {-1, -1, 0}, {1, -1, 0},  {0, 1, 1},   {0, -1, 1},  {0, 1, -1},  {0, -1, -1},
        {1, 0, 1},  {-1, 0, 1},  {1, 0, -1},  {-1, 0, -1}, {1, 1, 1},   {-1, 1, 1},  {-1, -1, 1},
        {1, -1, 1}, {1, 1, -1},  {-1, 1, -1}, {-1, -1, -1}, {1, -1, -1}};
    DBuf<int> derr;
    if (int rc = derr.alloc(ctx, 1)) return rc;
    MT_CUDA(ctx, cudaMemsetAsync(derr.p, 0, sizeof(int), ctx.stream));
    Box dom{{0, 0, 0}, {sp.coarse[0], sp.coarse[1], sp.coarse[2]}};
    // refinement regions (has_refine == 2) on the device; rbox[l]: the box of
    // level l's cells refined to l + 1, in level-l cells
    DBuf<uint8_t> dreg[MT_MAX_LEVELS + 1];
    Box rbox[MT_MAX_LEVELS];
    for (int l = 0; l < L; ++l) {
        if (sp.has_refine[l] == 2) {
            const std::vector<uint8_t> &h = c.h_reg[l + 1];
            if (int rc = dreg[l + 1].alloc(ctx, (int64_t)h.size())) return rc;
            MT_CUDA(ctx, cudaMemcpyAsync(dreg[l + 1].p, h.data(), h.size(), cudaMemcpyHostToDevice, ctx.stream));
            for (int a = 0; a < 3; ++a) {
                rbox[l].lo[a] = c.reg_lo[l + 1][a];
                rbox[l].hi[a] = c.reg_lo[l + 1][a] + c.reg_n[l + 1][a];
            }
        } else {
            for (int a = 0; a < 3; ++a) {
                rbox[l].lo[a] = sp.refine_lo[l][a];
                rbox[l].hi[a] = sp.refine_hi[l][a];
            }
        }
    }
    auto region = [&](int l) {  // the mask of level l's refined cells (l + 1's region)
        RegionMask r{dreg[l + 1].p, {0, 0, 0}, {0, 0, 0}};
        for (int a = 0; a < 3; ++a) {
            r.lo[a] = c.reg_lo[l + 1][a];
            r.n[a] = c.reg_n[l + 1][a];
        }
        return r;
    };
    SurfaceTables st;
    if (sp.sphere == 3) {
        if (L == 0) return set_err(ctx, MT_ERR_MESH, "the solid boundary is only applied on a refined finest level");
        Box f = dom;
        for (int l = 0; l < L; ++l) {
            Box nx{{0, 0, 0}, {0, 0, 0}};
            if (sp.has_refine[l] && f.n() > 0)
                for (int a = 0; a < 3; ++a) {
                    nx.lo[a] = 2 * rbox[l].lo[a];
                    nx.hi[a] = 2 * rbox[l].hi[a];
                }
            f = nx;
        }
        if (int rc = surface_tables(ctx, c.h_tri, L, f, st)) return rc;
    }
    for (int l = 0; l <= L; ++l) {
        LevelGen g{};
        g.level = l;
        g.L = L;
        g.q = q;
        for (int a = 0; a < 3; ++a) {
            g.ext[a] = sp.coarse[a] << l;
            g.bc[a] = sp.boundary_bc[a];
            g.per[a] = !sp.boundary_bc[a];
        }
        for (int i = 0; i < 27; ++i) g.side_bc[i] = -1;
        for (int b = 0; b < 26; ++b)
            g.side_bc[(sides[b][0] + 1) + 3 * (sides[b][1] + 1) + 9 * (sides[b][2] + 1)] = (int8_t)b;
        g.dom = dom;
        g.dom_region = l > 0 && sp.has_refine[l - 1] == 2;
        if (g.dom_region) g.dreg = region(l - 1);
        g.has_ref = l < L && sp.has_refine[l] && dom.n() > 0;
        g.ref_region = g.has_ref && sp.has_refine[l] == 2;
        if (g.ref_region) g.rreg = region(l);
        if (g.has_ref)
            for (int a = 0; a < 3; ++a) {
                g.ref.lo[a] = rbox[l].lo[a];
                g.ref.hi[a] = rbox[l].hi[a];
            }
        g.sphere = (l == L) ? sp.sphere : 0;
        const double s = (double)(1 << L);
        g.cx = sp.center[0] * s;
        g.cy = sp.center[1] * s;
        g.cz = sp.center[2] * s;
        g.r = sp.radius * s;
        g.amp = sp.osc_amplitude * s;
        g.slack = sp.band_slack * s;
        g.col_off = st.col_off.p;
        g.col_x = st.col_x.p;
        for (int a = 0; a < 2; ++a) {
            g.col_lo[a] = st.col_lo[a];
            g.col_n[a] = st.col_n[a];
        }
        if (g.sphere == 1 && L == 0)
            return set_err(ctx, MT_ERR_MESH, "the solid boundary is only applied on a refined finest level");
        Level &lv = c.lv[l];
        const int64_t nbox = dom.n();
        // next level's domain: the refinement box doubled
        Box next{{0, 0, 0}, {0, 0, 0}};
        if (g.has_ref)
            for (int a = 0; a < 3; ++a) {
                next.lo[a] = 2 * g.ref.lo[a];
                next.hi[a] = 2 * g.ref.hi[a];
            }
        dom = next;
        if (nbox <= 0) continue;
        // classify and sort the stored cells by key (not stored: ~0, last)
        DBuf<uint64_t> key, skey;
        DBuf<uint32_t> pay, spay;
        if (int rc = key.alloc(ctx, nbox)) return rc;
        if (int rc = pay.alloc(ctx, nbox)) return rc;
        if (int rc = skey.alloc(ctx, nbox)) return rc;
        if (int rc = spay.alloc(ctx, nbox)) return rc;
        k_classify<<<grid_for(nbox, 256), 256, 0, ctx.stream>>>(g, key.p, pay.p, derr.p);
        MT_LAUNCHED(ctx);
        {
            size_t tb = 0;
            MT_CUDA(ctx, cub::DeviceRadixSort::SortPairs(nullptr, tb, key.p, skey.p, pay.p, spay.p, (int)nbox, 0, 64,
                                                         ctx.stream));
            DBuf<char> tmp;
            if (int rc = tmp.alloc(ctx, (int64_t)tb)) return rc;
            MT_CUDA(ctx, cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.p, skey.p, pay.p, spay.p, (int)nbox, 0, 64,
                                                         ctx.stream));
        }
        // stored cells = keys below the sentinel
        int64_t ns = 0;
        {
            DBuf<uint64_t> all;
            DBuf<uint8_t> flag;
            if (int rc = flag.alloc(ctx, nbox)) return rc;
            k_member<<<grid_for(nbox, 256), 256, 0, ctx.stream>>>(skey.p, nbox, nullptr, 0, nullptr, 0, 0, flag.p);
            MT_LAUNCHED(ctx);
            if (int rc = select_flagged(ctx, skey.p, flag.p, nbox, all)) return rc;
            ns = all.n;
        }
        DBuf<uint64_t> latf, f2c, c2f, sf, band, gc2f, gf2c;
        if (int rc = set_keys(ctx, skey.p, spay.p, ns, 0, P_LATF, latf)) return rc;
        if (int rc = set_keys(ctx, skey.p, spay.p, ns, 0, P_F2C, f2c)) return rc;
        if (int rc = set_keys(ctx, skey.p, spay.p, ns, 0, P_C2F, c2f)) return rc;
        if (int rc = set_keys(ctx, skey.p, spay.p, ns, 0, P_SF, sf)) return rc;
        if (int rc = set_keys(ctx, skey.p, spay.p, ns, 1, 0, band)) return rc;
        if (l > 0 && c2f.n) {
            DBuf<uint64_t> cand, uniq;
            if (int rc = nbr_keys(ctx, g, c2f.p, c2f.n, cand)) return rc;
            if (int rc = sort_unique(ctx, cand.p, cand.n, uniq)) return rc;
            DBuf<uint8_t> flag;
            if (int rc = flag.alloc(ctx, uniq.n)) return rc;
            if (uniq.n) {
                k_member<<<grid_for(uniq.n, 256), 256, 0, ctx.stream>>>(uniq.p, uniq.n, latf.p, latf.n, c2f.p, c2f.n,
                                                                       0, flag.p);
                MT_LAUNCHED(ctx);
            }
            if (int rc = select_flagged(ctx, uniq.p, flag.p, uniq.n, gc2f)) return rc;
            if (gc2f.n) {
                k_check_in<<<grid_for(gc2f.n, 256), 256, 0, ctx.stream>>>(gc2f.p, gc2f.n, f2c.p, f2c.n, sf.p, sf.n,
                                                                         MERR_GHOST, derr.p);
                MT_LAUNCHED(ctx);
            }
        }
        if (l < L && f2c.n) {
            DBuf<uint64_t> cand, uniq;
            if (int rc = nbr_keys(ctx, g, f2c.p, f2c.n, cand)) return rc;
            if (int rc = sort_unique(ctx, cand.p, cand.n, uniq)) return rc;
            DBuf<uint8_t> flag;
            if (int rc = flag.alloc(ctx, uniq.n)) return rc;
            if (uniq.n) {
                k_member<<<grid_for(uniq.n, 256), 256, 0, ctx.stream>>>(uniq.p, uniq.n, latf.p, latf.n, nullptr, 0, 1,
                                                                       flag.p);
                MT_LAUNCHED(ctx);
            }
            if (int rc = select_flagged(ctx, uniq.p, flag.p, uniq.n, gf2c)) return rc;
        }
        if (l == L && (g.sphere == 1 || g.sphere == 3)) {
            // wall distances of the fluid cells; the solid must stay clear of C2F
            const int w = q - 1;
            DBuf<double> rows;
            DBuf<uint8_t> hit;
            if (int rc = rows.alloc(ctx, latf.n * w)) return rc;
            if (int rc = hit.alloc(ctx, latf.n)) return rc;
            if (latf.n && g.sphere == 1) {
                if (q == 19)
                    k_links<19><<<grid_for(latf.n, 128), 128, 0, ctx.stream>>>(latf.p, latf.n, g.cx, g.cy, g.cz, g.r,
                                                                              rows.p, hit.p);
                else
                    k_links<27><<<grid_for(latf.n, 128), 128, 0, ctx.stream>>>(latf.p, latf.n, g.cx, g.cy, g.cz, g.r,
                                                                              rows.p, hit.p);
                MT_LAUNCHED(ctx);
            } else if (latf.n) {
                if (q == 19)
                    k_links_surface<19><<<grid_for(latf.n, 128), 128, 0, ctx.stream>>>(
                        latf.p, latf.n, st.tri.p, st.box, st.bin_off.p, st.bin_tri.p, rows.p, hit.p);
                else
                    k_links_surface<27><<<grid_for(latf.n, 128), 128, 0, ctx.stream>>>(
                        latf.p, latf.n, st.tri.p, st.box, st.bin_off.p, st.bin_tri.p, rows.p, hit.p);
                MT_LAUNCHED(ctx);
            }
            // indices of the hit cells, in key order
            DBuf<int64_t> idx;
            DBuf<int> cnt;
            if (int rc = idx.alloc(ctx, latf.n)) return rc;
            if (int rc = cnt.alloc(ctx, 1)) return rc;
            int nd = 0;
            if (latf.n) {
                size_t tb = 0;
                cub::CountingInputIterator<int64_t> it(0);
                MT_CUDA(ctx, cub::DeviceSelect::Flagged(nullptr, tb, it, hit.p, idx.p, cnt.p, (int)latf.n, ctx.stream));
                DBuf<char> tmp;
                if (int rc = tmp.alloc(ctx, (int64_t)tb)) return rc;
                MT_CUDA(ctx, cub::DeviceSelect::Flagged(tmp.p, tb, it, hit.p, idx.p, cnt.p, (int)latf.n, ctx.stream));
                MT_CUDA(ctx, cudaMemcpyAsync(&nd, cnt.p, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
                MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
            }
            c.ndis = nd;
            if (nd) {
                MT_CUDA(ctx, cudaMallocAsync(&c.dis_key, 8 * (size_t)nd, ctx.stream));
                MT_CUDA(ctx, cudaMallocAsync(&c.dis, 8 * (size_t)nd * w, ctx.stream));
                k_gather_rows<<<grid_for((int64_t)nd * w, 256), 256, 0, ctx.stream>>>(idx.p, nd, rows.p, latf.p, w,
                                                                                      c.dis, c.dis_key);
                MT_LAUNCHED(ctx);
            }
            if (sf.n) {
                DBuf<uint64_t> nk;
                if (int rc = nbr_keys(ctx, g, sf.p, sf.n, nk)) return rc;
                k_check_in<<<grid_for(nk.n, 256), 256, 0, ctx.stream>>>(nk.p, nk.n, c2f.p, c2f.n, gc2f.p, gc2f.n,
                                                                       MERR_SOLID, derr.p);
                MT_LAUNCHED(ctx);
            }
        }
        if (l == L && g.sphere == 2 && band.n) {
            DBuf<uint64_t> nk;
            if (int rc = nbr_keys(ctx, g, band.p, band.n, nk)) return rc;
            k_check_in<<<grid_for(nk.n, 256), 256, 0, ctx.stream>>>(nk.p, nk.n, c2f.p, c2f.n, nullptr, 0, MERR_BAND,
                                                                   derr.p);
            MT_LAUNCHED(ctx);
        }
        // raw (key, set) pairs for the build: stored cells, the ghost layers, the band
        const int64_t nraw = ns + gc2f.n + gf2c.n + band.n;
        uint64_t *rk = nullptr;
        uint8_t *rs = nullptr;
        MT_CUDA(ctx, cudaMallocAsync(&rk, 8 * (size_t)std::max<int64_t>(nraw, 1), ctx.stream));
        MT_CUDA(ctx, cudaMallocAsync(&rs, (size_t)std::max<int64_t>(nraw, 1), ctx.stream));
        int64_t off = 0;
        if (ns) {
            MT_CUDA(ctx, cudaMemcpyAsync(rk, skey.p, 8 * ns, cudaMemcpyDeviceToDevice, ctx.stream));
            k_codes<<<grid_for(ns, 256), 256, 0, ctx.stream>>>(spay.p, ns, rs);
            MT_LAUNCHED(ctx);
            off = ns;
        }
        const DBuf<uint64_t> *extra[3] = {&gc2f, &gf2c, &band};
        const uint8_t codes[3] = {3, 4, (uint8_t)MT_SET_IB_BAND};
        for (int e = 0; e < 3; ++e) {
            const int64_t m = extra[e]->n;
            if (!m) continue;
            MT_CUDA(ctx, cudaMemcpyAsync(rk + off, extra[e]->p, 8 * m, cudaMemcpyDeviceToDevice, ctx.stream));
            k_fill_u8<<<grid_for(m, 256), 256, 0, ctx.stream>>>(rs + off, m, codes[e]);
            MT_LAUNCHED(ctx);
            off += m;
        }
        lv.draw_keys = rk;
        lv.draw_set = rs;
        lv.ndraw = nraw;
    }
    int herr = 0;
    MT_CUDA(ctx, cudaMemcpyAsync(&herr, derr.p, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    MT_CUDA(ctx, cudaStreamSynchronize(ctx.stream));
    if (herr & MERR_BOX_BC) return set_err(ctx, MT_ERR_MESH, "refinement box touches the boundary shell");
    if (herr & MERR_BOX_C2F) return set_err(ctx, MT_ERR_MESH, "refinement box too close to the coarse/fine interface");
    if (herr & MERR_GHOST) return set_err(ctx, MT_ERR_MESH, "ghost layer overlaps the next interface or the solid");
    if (herr & MERR_SOLID) return set_err(ctx, MT_ERR_MESH, "solid too close to the coarse/fine interface");
    if (herr & MERR_BAND) return set_err(ctx, MT_ERR_MESH, "the forcing band is too close to the coarse/fine interface");
    c.dis_on_device = true;
    return MT_OK;
}

}  // namespace mt
