// Two cells per lane in lockstep.  Each FP32 value of the reduced-precision
// collision is a pair (cell A in .x, cell B in .y) held in a 64-bit register
// pair and operated on by the sm_100 packed FP32 instructions (fma / add /
// mul on f32x2): one issue slot does both cells' arithmetic, which halves
// the instruction count of the collision, the part of the fused brick pass
// that bounds it.  Same operations as the scalar FP32 path (mt_lattice.cuh),
// with the FMA contractions written out, a multiply by 1/3 in place of the
// division by 3, and the moments the relaxation zeroes left out of the
// backward transform.
#pragma once

#include <cuda_runtime.h>

#include "mt_lattice.cuh"

namespace mt {
namespace p2 {

__device__ __forceinline__ float2 bc(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 neg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 sub(float2 a, float2 b) { return __fadd2_rn(a, neg(b)); }
__device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// 1 / rho with the reference's floor |rho| >= 1e-6 (SAFE_IRHO, Collision_Cumulant.cpp:17-20)
__device__ __forceinline__ float safe_inv(float r)
{
    return 1.f / ((r > -1e-6f && r < 1e-6f) ? ((r < 0.f) ? -1e-6f : 1e-6f) : r);
}
__device__ __forceinline__ float2 safe_inv(float2 r) { return make_float2(safe_inv(r.x), safe_inv(r.y)); }

// rho and velocity of both cells (LBM_Manager::calculateMacros, LBM_Manager.cpp:983-1001)
template <int Q> __device__ __forceinline__ void macros(const float2 *d, float2 &rho, float2 &ux, float2 &uy, float2 &uz)
{
    float2 r = d[0], vx = bc(0.f), vy = bc(0.f), vz = bc(0.f);
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        r = add(r, d[i]);
        if (ex(i) > 0) vx = add(vx, d[i]);
        if (ex(i) < 0) vx = sub(vx, d[i]);
        if (ey(i) > 0) vy = add(vy, d[i]);
        if (ey(i) < 0) vy = sub(vy, d[i]);
        if (ez(i) > 0) vz = add(vz, d[i]);
        if (ez(i) < 0) vz = sub(vz, d[i]);
    }
    rho = r;
    const float2 is = safe_inv(r);
    ux = mul(vx, is);
    uy = mul(vy, is);
    uz = mul(vz, is);
}

// e_k . u with the lattice constants folded
template <int Q> __device__ __forceinline__ float2 eu(int k, float2 x, float2 y, float2 z)
{
    float2 s = bc(0.f);
    bool any = false;
    auto acc = [&](int e, float2 v) {
        if (e == 0) return;
        if (!any) {
            s = e > 0 ? v : neg(v);
            any = true;
        } else {
            s = e > 0 ? add(s, v) : sub(s, v);
        }
    };
    acc(ex(k), x);
    acc(ey(k), y);
    acc(ez(k), z);
    return s;
}

// Collision_LBGK::collide on the stored deviations (the scalar path of
// collide_store): out_k = s_k + omega (feq_k - shift_k - s_k), s_k = d_k - shift_k
template <int Q>
__device__ __forceinline__ void lbgk(const float2 *d, float2 r, float2 x, float2 y, float2 z, float om, const Shift &sh,
                                     float2 *out)
{
    const float2 nuu = mul(bc(-1.5f), fma(x, x, fma(y, y, mul(z, z))));
    const float2 rm1 = sub(r, bc(1.f));
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const float2 e = eu<Q>(k, x, y, z);
        const float2 poly = (ex(k) | ey(k) | ez(k)) ? fma(e, fma(e, bc(4.5f), bc(3.f)), nuu) : nuu;
        const float2 dfeq = fma(bc((float)w<Q>(k)), fma(r, poly, rm1), bc(-sh.dw[k]));
        const float2 s = sub(d[k], bc(sh.v[k]));
        out[k] = fma(bc(om), sub(dfeq, s), s);
    }
}

// backward chimera step of one line (chim_back's FP32 polynomials); Z0, Z1,
// Z2 mark inputs known to be zero
template <bool Z0, bool Z1, bool Z2>
__device__ __forceinline__ void chim_back(float2 a0, float2 a1, float2 a2, float2 v, float2 tv, float2 v2, float2 &pn,
                                          float2 &pz, float2 &pp)
{
    float2 t, hh;
    if (Z0) {
        t = Z2 ? mul(tv, a1) : fma(tv, a1, a2);
        hh = a1;
    } else {
        const float2 inner = Z1 ? a2 : (Z2 ? mul(tv, a1) : fma(tv, a1, a2));
        t = (Z1 && Z2) ? mul(a0, v2) : fma(a0, v2, inner);
        hh = Z1 ? mul(a0, v) : fma(a0, v, a1);
    }
    const float2 h = mul(hh, bc(0.5f));
    pz = Z0 ? neg(t) : sub(a0, t);
    pp = fma(t, bc(0.5f), h);
    pn = fma(t, bc(0.5f), neg(h));
}

// D3Q27 cumulant collision of both cells (cumulant_collide's FP32 path,
// Collision_Cumulant.cpp:320-652): forward central moments by x, y, z
// chimera passes, second-order cumulants relaxed with omega1 and bulk rate 1,
// higher cumulants zero, backward transform.  The (2,1,0), (1,0,2), (0,2,1)
// moments keep their forward values (Collision_Cumulant.cpp:451-454).
__device__ __forceinline__ void cumulant(const float2 *f, float2 rho, float2 ux, float2 uy, float2 uz, float om1,
                                         float2 *out)
{
    float2 g[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) g[(ex(i) + 1) + 3 * (ey(i) + 1) + 9 * (ez(i) + 1)] = f[i];
    const float2 vel[3] = {ux, uy, uz};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int st = ax == 0 ? 1 : (ax == 1 ? 3 : 9);
        const float2 u = vel[ax], u2 = mul(u, u), mu = neg(u), m2u = mul(u, bc(-2.f));
#pragma unroll
        for (int line = 0; line < 9; ++line) {
            const int o1 = line % 3, o2 = line / 3;
            const int b = ax == 0 ? 3 * o1 + 9 * o2 : (ax == 1 ? o1 + 9 * o2 : o1 + 3 * o2);
            const float2 fm = g[b], f0 = g[b + st], fp = g[b + 2 * st];
            const float2 s1 = add(fp, fm), d1 = sub(fp, fm), k0 = add(s1, f0);
            g[b] = k0;
            g[b + st] = fma(mu, k0, d1);
            g[b + 2 * st] = fma(u2, k0, fma(m2u, d1, s1));
        }
    }
#define G(a, b, c) g[(a) + 3 * (b) + 9 * (c)]
    const float2 k000 = G(0, 0, 0);
    float2 c200 = G(2, 0, 0), c020 = G(0, 2, 0), c002 = G(0, 0, 2);
    float2 c110 = G(1, 1, 0), c101 = G(1, 0, 1), c011 = G(0, 1, 1);
    const float2 ir = safe_inv(rho);
    const float2 om = bc(om1), omc = bc(1.f - om1);
    // dxu = -(om1 (2 c200 - c020 - c002) + (c200 + c020 + c002 - k000)) ir / 2
    const float2 s3 = add(c200, add(c020, c002));
    const float2 tA = fma(bc(3.f), c200, neg(s3));
    const float2 dxu = mul(fma(om, tA, sub(s3, k000)), mul(ir, bc(-0.5f)));
    const float2 k3 = mul(ir, bc(1.5f * om1));
    const float2 d20 = sub(c200, c020), d02 = sub(c200, c002);
    const float2 dyv = fma(k3, d20, dxu);
    const float2 dzw = fma(k3, d02, dxu);
    c110 = mul(c110, omc);
    c101 = mul(c101, omc);
    c011 = mul(c011, omc);
    const float2 ux2 = mul(ux, ux), uy2 = mul(uy, uy), uz2 = mul(uz, uz);
    const float2 ax_ = mul(ux2, dxu), ay_ = mul(uy2, dyv), az_ = mul(uz2, dzw);
    const float2 nrq = mul(rho, bc(-3.f * (1.f - 0.5f * om1)));
    const float2 x1 = fma(nrq, sub(ax_, ay_), mul(omc, d20));
    const float2 x2 = fma(nrq, sub(ax_, az_), mul(omc, d02));
    const float2 x3 = fma(mul(rho, bc(-1.5f)), add(ax_, add(ay_, az_)), k000);
    c200 = mul(add(x1, add(x2, x3)), bc(1.f / 3.f));
    c020 = sub(c200, x1);
    c002 = sub(c200, x2);
    const float2 m210 = G(2, 1, 0), m102 = G(1, 0, 2), m021 = G(0, 2, 1);
    const float2 two = bc(2.f);
    const float2 m211 = mul(fma(c200, c011, mul(two, mul(c110, c101))), ir);
    const float2 m121 = mul(fma(c020, c101, mul(two, mul(c011, c110))), ir);
    const float2 m112 = mul(fma(c002, c110, mul(two, mul(c101, c011))), ir);
    const float2 m220 = mul(fma(c200, c020, mul(two, mul(c110, c110))), ir);
    const float2 m022 = mul(fma(c020, c002, mul(two, mul(c011, c011))), ir);
    const float2 m202 = mul(fma(c002, c200, mul(two, mul(c101, c101))), ir);
    const float2 m122 = mul(fma(c020, m102, mul(two, mul(c101, m021))), ir);
    const float2 m212 = mul(fma(c002, m210, mul(two, mul(c110, m102))), ir);
    const float2 m221 = mul(fma(c200, m021, mul(two, mul(c011, m210))), ir);
    const float2 a = mul(fma(c200, m022, fma(c020, m202, fma(c002, m220,
                             mul(bc(4.f), fma(c011, m211, fma(c101, m121, mul(c110, m112))))))), ir);
    const float2 bq = fma(mul(bc(16.f), c110), mul(c101, c011),
                          fma(bc(4.f), fma(mul(c101, c101), c020, fma(mul(c011, c011), c200, mul(mul(c110, c110), c002))),
                              mul(mul(two, c200), mul(c020, c002))));
    const float2 m222 = sub(a, mul(bq, mul(ir, ir)));
    // backward chimera, x lines (b, c) with (a0, a1, a2) = moments (0|1|2, b, c)
    float2 p1[27], p2[27];
    const float2 tvx = add(ux, ux);
    const float2 zero = bc(0.f);
    chim_back<false, false, false>(k000, G(1, 0, 0), c200, ux, tvx, ux2, p1[0], p1[1], p1[2]);
    chim_back<false, false, false>(G(0, 1, 0), c110, m210, ux, tvx, ux2, p1[3], p1[4], p1[5]);
    chim_back<false, true, false>(c020, zero, m220, ux, tvx, ux2, p1[6], p1[7], p1[8]);        // (1,2,0) = 0
    chim_back<false, false, true>(G(0, 0, 1), c101, zero, ux, tvx, ux2, p1[9], p1[10], p1[11]); // (2,0,1) = 0
    chim_back<false, true, false>(c011, zero, m211, ux, tvx, ux2, p1[12], p1[13], p1[14]);     // (1,1,1) = 0
    chim_back<false, false, false>(m021, m121, m221, ux, tvx, ux2, p1[15], p1[16], p1[17]);
    chim_back<false, false, false>(c002, m102, m202, ux, tvx, ux2, p1[18], p1[19], p1[20]);
    chim_back<true, false, false>(zero, m112, m212, ux, tvx, ux2, p1[21], p1[22], p1[23]);     // (0,1,2) = 0
    chim_back<false, false, false>(m022, m122, m222, ux, tvx, ux2, p1[24], p1[25], p1[26]);
    const float2 tvy = add(uy, uy), tvz = add(uz, uz);
#pragma unroll
    for (int ix = 0; ix < 3; ++ix)
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
            chim_back<false, false, false>(p1[ix + 9 * cc], p1[ix + 3 + 9 * cc], p1[ix + 6 + 9 * cc], uy, tvy, uy2,
                                           p2[ix + 9 * cc], p2[ix + 3 + 9 * cc], p2[ix + 6 + 9 * cc]);
#pragma unroll
    for (int ix = 0; ix < 3; ++ix)
#pragma unroll
        for (int iy = 0; iy < 3; ++iy)
            chim_back<false, false, false>(p2[ix + 3 * iy], p2[ix + 3 * iy + 9], p2[ix + 3 * iy + 18], uz, tvz, uz2,
                                           g[ix + 3 * iy], g[ix + 3 * iy + 9], g[ix + 3 * iy + 18]);
#undef G
#pragma unroll
    for (int i = 0; i < 27; ++i) out[i] = g[(ex(i) + 1) + 3 * (ey(i) + 1) + 9 * (ez(i) + 1)];
}

}  // namespace p2
}  // namespace mt
