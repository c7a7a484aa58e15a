// Lattice tables, Morton neighbour arithmetic and per-cell collision physics
// shared by every kernel of the library.
//
// Direction order, weights and inverse table: header/Constants.h:492-538 and
// LBM_Manager.cpp:137-169 of the reference.  The FP64 functions keep the
// reference's expression order so that, compiled without FMA contraction,
// they reproduce its results bit-for-bit; the FP32 variants are written for
// throughput (FMA, reciprocal of tau) and are compared against the FP64 path
// within stated tolerances.
#pragma once

#include <cstdint>
#include <type_traits>

#ifndef MT_HD
#define MT_HD __host__ __device__ __forceinline__
#endif

namespace mt {

MT_HD constexpr int ex(int k)
{
    constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, -1, 1};
    return t[k];
}
MT_HD constexpr int ey(int k)
{
    constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, 1, -1};
    return t[k];
}
MT_HD constexpr int ez(int k)
{
    constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1};
    return t[k];
}
MT_HD constexpr int inv(int k)
{
    constexpr int t[27] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};
    return t[k];
}
template <int Q> MT_HD constexpr double w(int k)
{
    return Q == 19 ? (k == 0 ? 1. / 3. : (k <= 6 ? 1. / 18. : 1. / 36.))
                   : (k == 0 ? 8. / 27. : (k <= 6 ? 2. / 27. : (k <= 18 ? 1. / 54. : 1. / 216.)));
}
// Storage shift of the reduced storages (FP32, FP16, BF16): they keep
// f_k - s_k with s_k = feq_k(1, u_s) = w_k (1 + 3 e.u_s + 4.5 (e.u_s)^2 -
// 1.5 u_s^2), so the stored deviations are small where the flow is near u_s
// (u_s = 0: s_k = w_k).  v: s_k rounded to FP32 (the compute type), dw: s_k -
// w_k rounded to FP32, d: s_k in FP64 (conversions from FP64 values), u: u_s.
// Kernels take it by value: with the direction loops unrolled its entries are
// constant-bank operands, as the literal weights were.
struct Shift {
    float v[27];
    float dw[27];
    float u[3];
    double d[27];
};
inline Shift make_shift(int q, const double *us)
{
    Shift s{};
    const double uu = us[0] * us[0] + us[1] * us[1] + us[2] * us[2];
    for (int k = 0; k < q; ++k) {
        const double wk = q == 19 ? w<19>(k) : w<27>(k);
        const double eu = ex(k) * us[0] + ey(k) * us[1] + ez(k) * us[2];
        const double dw = wk * (3.0 * eu + 4.5 * eu * eu - 1.5 * uu);
        s.d[k] = wk + dw;
        s.v[k] = (float)s.d[k];
        s.dw[k] = (float)dw;
    }
    for (int a = 0; a < 3; ++a) s.u[a] = (float)us[a];
    return s;
}

// D3Q19 weights used by the solid-boundary treatment for every Q; entries
// 19..26 are zero (ComplexBoundary_Manager.cpp:102-107,184-189).
MT_HD constexpr double w19z(int k) { return k >= 19 ? 0.0 : w<19>(k); }

// ---------------------------------------------------------------------------
// Morton keys.  A level-l cell at (x, y, z) in level-l units has the key
// interleave(x << (L-l), y << (L-l), z << (L-l)), x at bit 3i (Morton_Assist.cpp
// :185-193).  Neighbour steps are the reference's masked increment/decrement
// (Morton_Assist.h:229-289); a periodic axis wraps instead.
// ---------------------------------------------------------------------------
struct MortonGeom {
    int L;
    int periodic[3];
    int64_t extent0[3];
};

MT_HD uint64_t axis_mask(int L, int level, int axis)
{
    uint64_t m = 0;
    for (int k = L - level; k < 21; ++k) m |= (uint64_t)1 << (3 * k + axis);
    return m;
}
MT_HD uint64_t compact3(uint64_t v)
{
    v &= 0x1249249249249249ULL;
    v = (v ^ (v >> 2)) & 0x10C30C30C30C30C3ULL;
    v = (v ^ (v >> 4)) & 0x100F00F00F00F00FULL;
    v = (v ^ (v >> 8)) & 0x1F0000FF0000FFULL;
    v = (v ^ (v >> 16)) & 0x1F00000000FFFFULL;
    v = (v ^ (v >> 32)) & 0x1FFFFFULL;
    return v;
}
MT_HD uint64_t dilate3(uint64_t v)
{
    v &= 0x1FFFFFULL;
    v = (v | (v << 32)) & 0x1F00000000FFFFULL;
    v = (v | (v << 16)) & 0x1F0000FF0000FFULL;
    v = (v | (v << 8)) & 0x100F00F00F00F00FULL;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ULL;
    v = (v | (v << 2)) & 0x1249249249249249ULL;
    return v;
}
MT_HD uint64_t axis_step(const MortonGeom &g, uint64_t key, int level, int axis, int dir)
{
    const int L = g.L;
    const uint64_t m1 = axis_mask(L, level, axis);
    uint64_t others = 0;
    for (int a = 0; a < 3; ++a)
        if (a != axis) others |= key & axis_mask(L, level, a);
    if (g.periodic[axis]) {
        const int64_t ext = g.extent0[axis] << level;
        const int sh = L - level;
        int64_t c = (int64_t)(compact3(key >> axis) >> sh) + dir;
        if (c < 0) c += ext;
        if (c >= ext) c -= ext;
        return ((dilate3((uint64_t)c << sh) << axis) & m1) | others;
    }
    const int low = 3 * (L - level);
    const uint64_t one = (uint64_t)1 << (low + axis);
    uint64_t t;
    if (dir > 0) {
        uint64_t fill = ~m1;
        if (low > 0) fill &= ~(((uint64_t)1 << low) - 1);
        t = (key | fill) + one;
    } else {
        t = (key & m1) - one;
    }
    return (t & m1) | others;
}
MT_HD uint64_t find_neighbor(const MortonGeom &g, uint64_t key, int level, int dx, int dy, int dz)
{
    uint64_t r = key;
    if (dx) r = axis_step(g, r, level, 0, dx);
    if (dy) r = axis_step(g, r, level, 1, dy);
    if (dz) r = axis_step(g, r, level, 2, dz);
    return r;
}
MT_HD int64_t lower_bound_u64(const uint64_t *k, int64_t n, uint64_t key)
{
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = lo + ((hi - lo) >> 1);
        if (k[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}
MT_HD int64_t find_key(const uint64_t *k, int64_t n, uint64_t key)
{
    int64_t i = lower_bound_u64(k, n, key);
    return (i < n && k[i] == key) ? i : -1;
}

// ---------------------------------------------------------------------------
// FP64 physics in the reference's operation order
// ---------------------------------------------------------------------------
// LBM_Manager::calculateMacros(ddf, rho, v) (LBM_Manager.cpp:983-1001)
template <int Q> MT_HD void macros_ref(const double *d, double &rho, double &ux, double &uy, double &uz)
{
    double r = d[0], vx = 0., vy = 0., vz = 0.;
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        r += d[i];
        vx += d[i] * ex(i);
        vy += d[i] * ey(i);
        vz += d[i] * ez(i);
    }
    const double s = (r > -1e-6 && r < 1e-6) ? ((r < 0.0) ? -1e-6 : 1e-6) : r;
    rho = r;
    ux = vx / s;
    uy = vy / s;
    uz = vz / s;
}
// LBM_Manager::calculateFeq (BGK), one direction (LBM_Manager.cpp:205-233)
template <int Q> MT_HD double feq_ref(int i, double rho, double ux, double uy, double uz)
{
    const double uu = ux * ux + uy * uy + uz * uz;
    const double euv = ex(i) * ux + ey(i) * uy + ez(i) * uz;
    return rho * w<Q>(i) * (1. + 3. * euv + 4.5 * euv * euv - 1.5 * uu);
}
// LBM_Manager::calculateFeq_HeLuo, one direction (LBM_Manager.cpp:235-263)
template <int Q> MT_HD double feq_heluo_ref(int i, double rho, double ux, double uy, double uz)
{
    const double uu = ux * ux + uy * uy + uz * uz;
    const double euv = ex(i) * ux + ey(i) * uy + ez(i) * uz;
    return w<Q>(i) * (rho + 1.0 * (3. * euv + 4.5 * euv * euv - 1.5 * uu));
}

MT_HD double safe_irho_ref(double r) { return 1.0 / ((r > -1e-6 && r < 1e-6) ? ((r < 0.0) ? -1e-6 : 1e-6) : r); }

// The same three functions for any real type R: with R = double they are
// the reference-order versions above, with R = float the reduced-precision
// path's arithmetic.
template <int Q, class R> MT_HD void macros_g(const R *d, R &rho, R &ux, R &uy, R &uz)
{
    R r = d[0], vx = 0, vy = 0, vz = 0;
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        r += d[i];
        vx += d[i] * ex(i);
        vy += d[i] * ey(i);
        vz += d[i] * ez(i);
    }
    const R s = (r > R(-1e-6) && r < R(1e-6)) ? ((r < R(0)) ? R(-1e-6) : R(1e-6)) : r;
    rho = r;
    if constexpr (std::is_same<R, double>::value) {
        ux = vx / s;
        uy = vy / s;
        uz = vz / s;
    } else {
        const R is = R(1) / s;
        ux = vx * is;
        uy = vy * is;
        uz = vz * is;
    }
}
template <int Q, class R> MT_HD R feq_g(int i, R rho, R ux, R uy, R uz)
{
    const R uu = ux * ux + uy * uy + uz * uz;
    const R euv = ex(i) * ux + ey(i) * uy + ez(i) * uz;
    return rho * (R)w<Q>(i) * (R(1) + R(3) * euv + R(4.5) * euv * euv - R(1.5) * uu);
}
template <int Q, class R> MT_HD R feq_heluo_g(int i, R rho, R ux, R uy, R uz)
{
    const R uu = ux * ux + uy * uy + uz * uz;
    const R euv = ex(i) * ux + ey(i) * uy + ez(i) * uz;
    return (R)w<Q>(i) * (rho + R(1) * (R(3) * euv + R(4.5) * euv * euv - R(1.5) * uu));
}

template <class R>
MT_HD void chim_back(R a0, R a1, R a2, R v, R v2, R &pn, R &pz, R &pp)
{
    if constexpr (std::is_same<R, double>::value) {
        // the reference's expression order (Collision_Cumulant.cpp:486-651)
        pz = a0 * (1 - v2) - a1 * 2 * v - a2;
        pn = (a0 * (v2 - v) + a1 * (2 * v - 1) + a2) * R(0.5);
        pp = (a0 * (v2 + v) + a1 * (2 * v + 1) + a2) * R(0.5);
    } else {
        // the same polynomials with shared terms: t = a0 v^2 + 2 v a1 + a2,
        // h = (a0 v + a1) / 2; pz = a0 - t, pp = t / 2 + h, pn = t / 2 - h
        const R t = a0 * v2 + (2 * v * a1 + a2);
        const R h = R(0.5) * (a0 * v + a1);
        pz = a0 - t;
        pp = R(0.5) * t + h;
        pn = R(0.5) * t - h;
    }
}

// D3Q27 cumulant collision (Collision_Cumulant.cpp:320-652): central moments
// about u, second-order cumulants relaxed with omega1 = 1/tau and bulk rate 1,
// all cumulants of order >= 3 reset to zero, backward cumulant and chimera
// transforms.  Slot (a,b,c) of the moment arrays is a + 3b + 9c.  The
// (2,1,0), (1,0,2) and (0,2,1) moments keep their forward values in the
// backward pass, as in the reference (Collision_Cumulant.cpp:451-454).
// R = double reproduces the reference bit-for-bit without FMA contraction;
// R = float is the reduced-precision variant.
// The part of cumulant_collide after the forward central moments: cumulant
// relaxation and the backward transforms (Collision_Cumulant.cpp:374-652);
// m holds the 27 central moments about u, slot (a,b,c) = a + 3b + 9c, and is
// overwritten.
template <class R>
MT_HD void cumulant_from_moments(R *m, R rho, R ux, R uy, R uz, R omega1, R *out)
{
#define MM(a, b, c) m[(a) + 3 * (b) + 9 * (c)]
    R c200 = MM(2, 0, 0), c020 = MM(0, 2, 0), c002 = MM(0, 0, 2);
    R c110 = MM(1, 1, 0), c101 = MM(1, 0, 1), c011 = MM(0, 1, 1);
    const R k000 = MM(0, 0, 0);
    const R om1 = omega1, om2 = 1;
    const R ir = R(1) / ((rho > R(-1e-6) && rho < R(1e-6)) ? ((rho < R(0)) ? R(-1e-6) : R(1e-6)) : rho);
    const R dxu = -(om1 * (2 * c200 - c020 - c002) + om2 * (c200 + c020 + c002 - k000)) * ir * R(0.5);
    const R dyv = dxu + 3 * om1 * (c200 - c020) * R(0.5) * ir;
    const R dzw = dxu + 3 * om1 * (c200 - c002) * R(0.5) * ir;
    c110 *= (1 - om1);
    c101 *= (1 - om1);
    c011 *= (1 - om1);
    const R ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
    const R x1 = (1 - om1) * (c200 - c020) - 3 * rho * (1 - om1 * R(0.5)) * (ux2 * dxu - uy2 * dyv);
    const R x2 = (1 - om1) * (c200 - c002) - 3 * rho * (1 - om1 * R(0.5)) * (ux2 * dxu - uz2 * dzw);
    const R x3 = k000 * om2 + (1 - om2) * (c200 + c020 + c002) -
                 3 * rho * (1 - om2 * R(0.5)) * (ux2 * dxu + uy2 * dyv + uz2 * dzw);
    if constexpr (std::is_same<R, double>::value)
        c200 = (x1 + x2 + x3) / 3;  // the reference's expression
    else
        c200 = (x1 + x2 + x3) * R(1.0 / 3.0);
    c020 = c200 - x1;
    c002 = c200 - x2;

    MM(1, 1, 0) = c110; MM(0, 1, 1) = c011; MM(1, 0, 1) = c101;
    MM(2, 0, 0) = c200; MM(0, 2, 0) = c020; MM(0, 0, 2) = c002;
    MM(1, 2, 0) = 0; MM(0, 1, 2) = 0; MM(2, 0, 1) = 0;
    MM(1, 1, 1) = 0;
    MM(2, 1, 1) = 0 + (MM(2, 0, 0) * MM(0, 1, 1) + 2 * MM(1, 1, 0) * MM(1, 0, 1)) * ir;
    MM(1, 2, 1) = 0 + (MM(0, 2, 0) * MM(1, 0, 1) + 2 * MM(0, 1, 1) * MM(1, 1, 0)) * ir;
    MM(1, 1, 2) = 0 + (MM(0, 0, 2) * MM(1, 1, 0) + 2 * MM(1, 0, 1) * MM(0, 1, 1)) * ir;
    MM(2, 2, 0) = 0 + (MM(2, 0, 0) * MM(0, 2, 0) + 2 * MM(1, 1, 0) * MM(1, 1, 0)) * ir;
    MM(0, 2, 2) = 0 + (MM(0, 2, 0) * MM(0, 0, 2) + 2 * MM(0, 1, 1) * MM(0, 1, 1)) * ir;
    MM(2, 0, 2) = 0 + (MM(0, 0, 2) * MM(2, 0, 0) + 2 * MM(1, 0, 1) * MM(1, 0, 1)) * ir;
    MM(1, 2, 2) = 0 + (MM(0, 0, 2) * MM(1, 2, 0) + MM(0, 2, 0) * MM(1, 0, 2) + 4 * MM(0, 1, 1) * MM(1, 1, 1) +
                       2 * (MM(1, 0, 1) * MM(0, 2, 1) + MM(1, 1, 0) * MM(0, 1, 2))) * ir;
    MM(2, 1, 2) = 0 + (MM(2, 0, 0) * MM(0, 1, 2) + MM(0, 0, 2) * MM(2, 1, 0) + 4 * MM(1, 0, 1) * MM(1, 1, 1) +
                       2 * (MM(1, 1, 0) * MM(1, 0, 2) + MM(0, 1, 1) * MM(2, 0, 1))) * ir;
    MM(2, 2, 1) = 0 + (MM(0, 2, 0) * MM(2, 0, 1) + MM(2, 0, 0) * MM(0, 2, 1) + 4 * MM(1, 1, 0) * MM(1, 1, 1) +
                       2 * (MM(0, 1, 1) * MM(2, 1, 0) + MM(1, 0, 1) * MM(1, 2, 0))) * ir;
    {
        const R a = (4 * MM(1, 1, 1) * MM(1, 1, 1) + MM(2, 0, 0) * MM(0, 2, 2) + MM(0, 2, 0) * MM(2, 0, 2) +
                     MM(0, 0, 2) * MM(2, 2, 0) +
                     4 * (MM(0, 1, 1) * MM(2, 1, 1) + MM(1, 0, 1) * MM(1, 2, 1) + MM(1, 1, 0) * MM(1, 1, 2)) +
                     2 * (MM(1, 2, 0) * MM(1, 0, 2) + MM(2, 1, 0) * MM(0, 1, 2) + MM(2, 0, 1) * MM(0, 2, 1))) * ir;
        const R b = (16 * MM(1, 1, 0) * MM(1, 0, 1) * MM(0, 1, 1) +
                     4 * (MM(1, 0, 1) * MM(1, 0, 1) * MM(0, 2, 0) + MM(0, 1, 1) * MM(0, 1, 1) * MM(2, 0, 0) +
                          MM(1, 1, 0) * MM(1, 1, 0) * MM(0, 0, 2)) +
                     2 * MM(2, 0, 0) * MM(0, 2, 0) * MM(0, 0, 2)) * ir * ir;
        MM(2, 2, 2) = 0 + a - b;
    }
    R p1[27], p2[27];
    const R vx2 = ux * ux, vy2 = uy * uy, vz2 = uz * uz;
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            chim_back<R>(MM(0, b, cc), MM(1, b, cc), MM(2, b, cc), ux, vx2, p1[0 + 3 * b + 9 * cc],
                         p1[1 + 3 * b + 9 * cc], p1[2 + 3 * b + 9 * cc]);
#pragma unroll
    for (int ix = 0; ix < 3; ++ix)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
            chim_back<R>(p1[ix + 0 + 9 * cc], p1[ix + 3 + 9 * cc], p1[ix + 6 + 9 * cc], uy, vy2, p2[ix + 0 + 9 * cc],
                         p2[ix + 3 + 9 * cc], p2[ix + 6 + 9 * cc]);
#pragma unroll
    for (int ix = 0; ix < 3; ++ix)
#pragma unroll
        for (int iy = 0; iy < 3; ++iy)
            chim_back<R>(p2[ix + 3 * iy + 0], p2[ix + 3 * iy + 9], p2[ix + 3 * iy + 18], uz, vz2, m[ix + 3 * iy + 0],
                         m[ix + 3 * iy + 9], m[ix + 3 * iy + 18]);
#pragma unroll
    for (int i = 0; i < 27; ++i) out[i] = m[(ex(i) + 1) + 3 * (ey(i) + 1) + 9 * (ez(i) + 1)];
#undef MM
}

template <class R>
MT_HD void cumulant_collide(const R *f, R rho, R ux, R uy, R uz, R omega1, R *out)
{
    R m[27];
#define MM(a, b, c) m[(a) + 3 * (b) + 9 * (c)]
    if constexpr (!std::is_same<R, double>::value) {
        // reduced precision: the same central moments by three chimera passes
        // (x, then y, then z lines of three), a quarter of the operations
        R g[27];
#pragma unroll
        for (int i = 0; i < 27; ++i) g[(ex(i) + 1) + 3 * (ey(i) + 1) + 9 * (ez(i) + 1)] = f[i];
        const R v[3] = {ux, uy, uz};
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const int st = ax == 0 ? 1 : (ax == 1 ? 3 : 9);
            const R u = v[ax], u2 = u * u;
#pragma unroll
            for (int line = 0; line < 9; ++line) {
                // base index of the line: the two other axes' positions
                const int o1 = line % 3, o2 = line / 3;
                const int bidx = ax == 0 ? 3 * o1 + 9 * o2 : (ax == 1 ? o1 + 9 * o2 : o1 + 3 * o2);
                const R fm = g[bidx], f0 = g[bidx + st], fp = g[bidx + 2 * st];
                const R k0 = fm + f0 + fp, d1 = fp - fm, s1 = fp + fm;
                g[bidx] = k0;
                g[bidx + st] = d1 - u * k0;
                g[bidx + 2 * st] = s1 - 2 * u * d1 + u2 * k0;
            }
        }
#pragma unroll
        for (int i = 0; i < 27; ++i) m[i] = g[i];
    } else {
#pragma unroll
    for (int i = 0; i < 27; ++i) m[i] = 0;
#pragma unroll
    for (int i = 0; i < 27; ++i) {
        const R cx = ex(i) - ux, cy = ey(i) - uy, cz = ez(i) - uz, fi = f[i];
        MM(0, 0, 0) += fi;
        MM(1, 0, 0) += cx * fi;
        MM(0, 1, 0) += cy * fi;
        MM(0, 0, 1) += cz * fi;
        MM(2, 0, 0) += cx * cx * fi;
        MM(0, 2, 0) += cy * cy * fi;
        MM(0, 0, 2) += cz * cz * fi;
        MM(1, 1, 0) += cx * cy * fi;
        MM(1, 0, 1) += cx * cz * fi;
        MM(0, 1, 1) += cy * cz * fi;
        MM(2, 1, 0) += cx * cx * cy * fi;
        MM(2, 0, 1) += cx * cx * cz * fi;
        MM(0, 2, 1) += cy * cy * cz * fi;
        MM(1, 2, 0) += cx * cy * cy * fi;
        MM(1, 0, 2) += cx * cz * cz * fi;
        MM(0, 1, 2) += cy * cz * cz * fi;
        MM(1, 1, 1) += cx * cy * cz * fi;
        MM(2, 2, 0) += cx * cx * cy * cy * fi;
        MM(2, 0, 2) += cx * cx * cz * cz * fi;
        MM(0, 2, 2) += cy * cy * cz * cz * fi;
        MM(2, 1, 1) += cx * cx * cy * cz * fi;
        MM(1, 2, 1) += cx * cy * cy * cz * fi;
        MM(1, 1, 2) += cx * cy * cz * cz * fi;
        MM(2, 2, 1) += cx * cx * cy * cy * cz * fi;
        MM(2, 1, 2) += cx * cx * cy * cz * cz * fi;
        MM(1, 2, 2) += cx * cy * cy * cz * cz * fi;
        MM(2, 2, 2) += cx * cx * cy * cy * cz * cz * fi;
    }
    }
    cumulant_from_moments<R>(m, rho, ux, uy, uz, omega1, out);
#undef MM
}

// Reduced precision D3Q27 cumulant with the macroscopic moments taken from
// the collision's own first chimera pass: the populations are grouped into
// the nine x lines of three (e_x = -1, 0, +1) and summed along each line
// once; the line sums give rho and the momentum directly (rho = sum of the
// line totals k0, j_x = sum of the line differences d1, j_y / j_z = the line
// totals of the e_y / e_z = +1 lines minus those of the -1 lines), and the
// same sums are the x pass of the forward transform once u is known.  The
// rest is cumulant_collide's FP32 path.  Saves the separate macros pass over
// the 27 populations and the x pass's own line sums.
MT_HD void cumulant_macros_collide(const float *f, float &rho, float &ux, float &uy, float &uz, float omega1,
                                    float *out)
{
    float g[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) g[(ex(i) + 1) + 3 * (ey(i) + 1) + 9 * (ez(i) + 1)] = f[i];
    // x lines: slot 0 line total k0, slot 1 difference d1, slot 2 sum of the ends s1
    float r = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int line = 0; line < 9; ++line) {
        const int b = 3 * line;
        const float fm = g[b], f0 = g[b + 1], fp = g[b + 2];
        const float s1 = fp + fm, d1 = fp - fm, k0 = s1 + f0;
        g[b] = k0;
        g[b + 1] = d1;
        g[b + 2] = s1;
        r += k0;
        jx += d1;
        const int ly = line % 3, lz = line / 3;  // y, z positions 0 1 2 = -1 0 +1
        if (ly == 2) jy += k0;
        if (ly == 0) jy -= k0;
        if (lz == 2) jz += k0;
        if (lz == 0) jz -= k0;
    }
    const float is = 1.f / ((r > -1e-6f && r < 1e-6f) ? ((r < 0.f) ? -1e-6f : 1e-6f) : r);
    rho = r;
    ux = jx * is;
    uy = jy * is;
    uz = jz * is;
    {
        const float u = ux, u2 = u * u;
#pragma unroll
        for (int line = 0; line < 9; ++line) {
            const int b = 3 * line;
            const float k0 = g[b], d1 = g[b + 1], s1 = g[b + 2];
            g[b + 1] = d1 - u * k0;
            g[b + 2] = s1 - 2 * u * d1 + u2 * k0;
        }
    }
    const float v[3] = {ux, uy, uz};
#pragma unroll
    for (int ax = 1; ax < 3; ++ax) {
        const int st = ax == 1 ? 3 : 9;
        const float u = v[ax], u2 = u * u;
#pragma unroll
        for (int line = 0; line < 9; ++line) {
            const int o1 = line % 3, o2 = line / 3;
            const int bidx = ax == 1 ? o1 + 9 * o2 : o1 + 3 * o2;
            const float fm = g[bidx], f0 = g[bidx + st], fp = g[bidx + 2 * st];
            const float k0 = fm + f0 + fp, d1 = fp - fm, s1 = fp + fm;
            g[bidx] = k0;
            g[bidx + st] = d1 - u * k0;
            g[bidx + 2 * st] = s1 - 2 * u * d1 + u2 * k0;
        }
    }
    cumulant_from_moments<float>(g, rho, ux, uy, uz, omega1, out);
}

}  // namespace mt
