// Per-phase kernels of the multi-level time step, templated on the
// population storage type S (mt_store.cuh).  With S = double every
// expression keeps the reference's operation order and, compiled without
// FMA contraction (mt_amr_f64.cu), reproduces its results bit-for-bit; the
// float / half / bfloat16 instantiations (mt_amr_lp.cu) store f - s_q, s_q
// the level's storage shift (the weights unless set), and compute in FP32.
//
// Macros are computed inside the collision kernel from the same f the
// reference's calculateMacros(level) reads just before collide(level)
// (LBM_Simulator.cpp:26-28), and written out for the solid boundary and the
// domain boundary that read them later in the substep.
#pragma once

#include <algorithm>

#include "mt_internal.hpp"
#include "mt_pack2.cuh"
#include "mt_store.cuh"

namespace mt {


// reserved boundary directions; one copy per translation unit, uploaded by
// AmrOps<S>::upload_tables when a case of that storage type is built
static __constant__ int8_t c_bdry19[26][14];
static __constant__ int8_t c_bdry27[26][18];

template <int Q, class S>
__global__ void k_init_eq(int64_t n, const uint32_t *tag, double rho0, double ux, double uy, double uz, S *f, S *fcol,
                          typename Store<S>::C *rho, typename Store<S>::C *u, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = tag[i];
    const bool solid = (t & TAG_SF) && !(t & (TAG_LATF | TAG_F2C | TAG_C2F | TAG_GC2F | TAG_BC));
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double v = solid ? 0. : feq_ref<Q>(k, rho0, ux, uy, uz);
        const C s = stored_f64<S>(sh, v, k);
        T::st(f, k * n + i, s);
        T::st(fcol, k * n + i, s);
    }
    rho[i] = (C)(solid ? 1. : rho0);
    u[i] = (C)(solid ? 0. : ux);
    u[n + i] = (C)(solid ? 0. : uy);
    u[2 * n + i] = (C)(solid ? 0. : uz);
}

// LBM_Manager::calculateMacros(level), LBM_Manager.cpp:1003-1050
template <int Q, class S>
__global__ void k_macros(const int32_t *list, int64_t nl, int64_t n, const S *f, typename Store<S>::C *rho,
                         typename Store<S>::C *u, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    C d[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) d[k] = full_sh<S>(sh, T::ld(f, k * n + i), k);
    C r, x, y, z;
    macros_g<Q, C>(d, r, x, y, z);
    rho[i] = r;
    u[i] = x;
    u[n + i] = y;
    u[2 * n + i] = z;
}

// post-collision populations of one cell from its f (already in the compute
// type C) and its macros: Collision_LBGK::collide (Collision_Manager.cpp:13-53)
// or Collision_Cumulant::collide (Collision_Cumulant.cpp:22-159), stored into
// fcol[k * n + i].  Shared by the phase kernel and the fused pull + collide
// kernels so both schedules run the same arithmetic.
template <int Q, class S, int COLL, class I = int64_t>
__device__ __forceinline__ void collide_store(const typename Store<S>::C *d, typename Store<S>::C r,
                                              typename Store<S>::C x, typename Store<S>::C y,
                                              typename Store<S>::C z, double tau, S *fcol, I n, I i, const Shift &sh)
{
    using T = Store<S>;
    using C = typename T::C;
    if constexpr (COLL == MT_COLL_LBGK) {
        if constexpr (!T::shifted) {
#pragma unroll
            for (int k = 0; k < Q; ++k) {
                const double fk = d[k];
                fcol[(I)k * n + i] = fk - (fk - feq_ref<Q>(k, r, x, y, z)) / tau;
            }
        } else {
            const float om = (float)(1.0 / tau);
            const float uu = 1.5f * (x * x + y * y + z * z);
#pragma unroll
            for (int k = 0; k < Q; ++k) {
                const float eu = ex(k) * x + ey(k) * y + ez(k) * z;
                const float wk = (float)w<Q>(k);
                // deviations from the shift s_k = w_k + dw_k:
                // feq - s = w ((rho - 1) + rho (3 eu + 4.5 eu^2 - 1.5 u^2)) - dw
                const float dfeq = wk * ((r - 1.f) + r * (3.f * eu + 4.5f * eu * eu - uu)) - sh.dw[k];
                const float s = d[k] - sh.v[k];
                T::st(fcol, (I)k * n + i, fmaf(om, dfeq - s, s));
            }
        }
    } else if constexpr (Q == 27) {
        C o[27];
        cumulant_collide<C>(d, r, x, y, z, (C)(1. / tau), o);
#pragma unroll
        for (int k = 0; k < 27; ++k) T::st(fcol, (I)k * n + i, stored_sh<S>(sh, o[k], k));
    }
}

// The macros of d (rho, u into r, x, y, z) and its collision stored into
// out: the reduced-precision D3Q27 cumulant takes the macros from the
// collision's own first chimera pass (cumulant_macros_collide); every other
// form computes them with macros_g and then collides (collide_store).
template <int Q, class S, int COLL, class I>
__device__ __forceinline__ void macros_collide_store(const typename Store<S>::C *d, typename Store<S>::C &r,
                                                     typename Store<S>::C &x, typename Store<S>::C &y,
                                                     typename Store<S>::C &z, double tau, S *out, I n, I i,
                                                     const Shift &sh)
{
    using T = Store<S>;
    if constexpr (COLL == MT_COLL_CUMULANT && Q == 27 && T::shifted) {
        float o[27];
        cumulant_macros_collide(d, r, x, y, z, (float)(1. / tau), o);
#pragma unroll
        for (int k = 0; k < 27; ++k) T::st(out, (I)k * n + i, stored_sh<S>(sh, o[k], k));
    } else {
        macros_g<Q, typename T::C>(d, r, x, y, z);
        collide_store<Q, S, COLL>(d, r, x, y, z, tau, out, n, i, sh);
    }
}

// calculateMacros(level) + Collision_LBGK::collide / Collision_Cumulant::collide
// on lat_f then overlap_F2C (Collision_Manager.cpp:13-53, Collision_Cumulant.cpp:22-159)
template <int Q, class S, int COLL>
__global__ void k_collide(const int32_t *list, int64_t nl, int64_t n, double tau, const S *f,
                          typename Store<S>::C *rho, typename Store<S>::C *u, S *fcol, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    C d[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) d[k] = full_sh<S>(sh, T::ld(f, k * n + i), k);
    C r, x, y, z;
    macros_collide_store<Q, S, COLL>(d, r, x, y, z, tau, fcol, n, i, sh);
    rho[i] = r;
    u[i] = x;
    u[n + i] = y;
    u[2 * n + i] = z;
    
}

// fcol = f on overlap_C2F (Collision_Manager.cpp:45-52)
template <int Q, class S>
__global__ void k_copy_fcol(const int32_t *list, int64_t nl, int64_t n, const S *f, S *fcol)
{
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
#pragma unroll
    for (int k = 0; k < Q; ++k) fcol[k * n + i] = f[k * n + i];
}

// ABPatternPull::stream (Stream_Manager.cpp:43-76): a missing neighbour keeps f
template <int Q, class S>
__global__ void k_stream(const int32_t *list, int64_t nl, int64_t n, int textbook, const int32_t *nbr, const S *fcol,
                         S *f)
{
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
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

// AMR_transDDF_explosion (LBM_Manager.cpp:1059-1129), eight threads per
// coarse source cell, one per child: each computes the (identical) rescaled
// populations and writes its own child, so the eight children of a source
// (consecutive in key order) take one contiguous store per direction.
// With a second post-collision buffer (fused schedule) the children of ghost
// F2C cells (sources from nf2c on) are written to both: nothing else writes
// them, and the reference keeps them over the second substep.
// cprev (MT_ITIME_EXTRAP, second substep): the sources' parent values at the
// parent's previous step, [Q][ns]; the explosion then starts from
// 1.5 fcol - 0.5 prev, the parent state extrapolated to the half step.
template <int Q, class S>
__global__ void k_explosion(const int32_t *__restrict__ src, const int32_t *__restrict__ child, int64_t ns,
                            int64_t nc, const S *__restrict__ cfcol, int64_t nf, S *__restrict__ ffcol, double scale,
                            S *__restrict__ ffcol2, int64_t nf2c, const Shift csh, const Shift fsh,
                            const S *__restrict__ cprev = nullptr)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t j = t >> 3;
    const int m = (int)(t & 7);
    if (j >= ns) return;
    const int32_t ch = child[(int64_t)m * ns + j];
    if (ch < 0) return;
    const int64_t i = src[j];
    C d[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) d[k] = full_sh<S>(csh, T::ld(cfcol, k * nc + i), k);
    if (cprev) {
#pragma unroll
        for (int k = 0; k < Q; ++k) d[k] = C(1.5) * d[k] - C(0.5) * full_sh<S>(csh, T::ld(cprev, k * ns + j), k);
    }
    C r, x, y, z;
    macros_g<Q, C>(d, r, x, y, z);
    const bool both = ffcol2 && j >= nf2c;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const C fe = feq_heluo_g<Q, C>(k, r, x, y, z);
        const C v = stored_sh<S>(fsh, fe + (C)scale * (d[k] - fe), k);
        T::st(ffcol, k * nf + ch, v);
        if (both) T::st(ffcol2, k * nf + ch, v);
    }
}

// the explosion sources' parent values into prev [Q][ns] (MT_ITIME_EXTRAP)
template <int Q, class S>
__global__ void k_expl_save(const int32_t *__restrict__ src, int64_t ns, const S *__restrict__ cfcol, int64_t nc,
                            S *__restrict__ prev)
{
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= ns) return;
    const int64_t i = src[j];
#pragma unroll
    for (int k = 0; k < Q; ++k) prev[k * ns + j] = cfcol[k * nc + i];
}

// AMR_transDDF_coalescence (LBM_Manager.cpp:1131-1169)
template <int Q, class S>
__global__ void k_coalescence(const int32_t *list, const int32_t *child, int64_t nl, int64_t nc, S *cf, const S *ff,
                              int64_t nf, double scale, const Shift csh, const Shift fsh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    int32_t ch[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) ch[m] = child[(int64_t)m * nl + j];
    C a[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        C s = 0;
#pragma unroll
        for (int m = 0; m < 8; ++m) s += full_sh<S>(fsh, T::ld(ff, k * nf + ch[m]), k);
        a[k] = s / (C)8.0;
    }
    C r, x, y, z;
    macros_g<Q, C>(a, r, x, y, z);
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const C fe = feq_heluo_g<Q, C>(k, r, x, y, z);
        T::st(cf, k * nc + i, stored_sh<S>(csh, fe + (C)scale * (a[k] - fe), k));
    }
}

// Fused schedule: coalescence onto the F2C cells, then (the cells' f being
// untouched until the next substep's collide) their next collision into
// fnext, from the stored f as the reference's collide would read it; the
// macros of that f are written when `macros` is set (the level's last
// substep of the coarse step: calculateMacros of every level follows).
template <int Q, class S, int COLL>
__global__ void k_coal_collide(const int32_t *__restrict__ list, const int32_t *__restrict__ child, int64_t nl,
                               int64_t nc, S *__restrict__ cf, const S *__restrict__ ff, int64_t nf, double scale,
                               double tau, S *__restrict__ cfnext, typename Store<S>::C *__restrict__ rho,
                               typename Store<S>::C *__restrict__ u, int macros, const Shift csh,
                               const Shift fsh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    int32_t ch[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) ch[m] = child[(int64_t)m * nl + j];
    C a[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        C s = 0;
#pragma unroll
        for (int m = 0; m < 8; ++m) s += full_sh<S>(fsh, T::ld(ff, k * nf + ch[m]), k);
        a[k] = s / (C)8.0;
    }
    C r, x, y, z;
    macros_g<Q, C>(a, r, x, y, z);
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const C fe = feq_heluo_g<Q, C>(k, r, x, y, z);
        const C st = stored_sh<S>(csh, fe + (C)scale * (a[k] - fe), k);
        T::st(cf, k * nc + i, st);
        S sv;
        T::st(&sv, 0, st);
        a[k] = full_sh<S>(csh, T::cv(sv), k);
    }
    macros_collide_store<Q, S, COLL>(a, r, x, y, z, tau, cfnext, nc, i, csh);
    if (macros) {
        rho[i] = r;
        u[i] = x;
        u[nc + i] = y;
        u[2 * nc + i] = z;
    }
}

// Non-equilibrium extrapolation ("eflow stable" form) on one boundary set:
// f_k(b) = feq_k(rho_b, u_bc) + f_k(b + e_k) - feq_k(rho_n, u_n) over the
// reserved directions (NonEquilibrumExtrapolation.cpp:33-71).  Boundary f
// is read by nothing but this update: a Jacobi sweep (values first, then
// writes) keeps it deterministic.
template <int Q, class S>
__global__ void k_bc_neq(const int32_t *list, int64_t nl, int b, int64_t n, const int32_t *nbr,
                         const typename Store<S>::C *rho, const typename Store<S>::C *u, S *f, double ubx,
                         double uby, double ubz, double *tmp, int phase, int *err, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
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
                tmp[t * nl + j] = (double)full_sh<S>(sh, T::ld(f, k * n + i), k);
                continue;
            }
            const C fw = feq_g<Q, C>(k, rho[i], (C)ubx, (C)uby, (C)ubz);
            const C fn = feq_g<Q, C>(k, rho[nb], u[nb], u[n + nb], u[2 * n + nb]);
            tmp[t * nl + j] = (double)(fw + full_sh<S>(sh, T::ld(f, k * n + nb), k) - fn);
        } else {
            T::st(f, k * n + i, stored_sh<S>(sh, (C)tmp[t * nl + j], k));
        }
    }
}

// the same sweep over every boundary set at once (one Jacobi pass: all values,
// then all writes); setb gives each cell's set, ub its face's velocity
struct BcVel {
    double u[26][3];
};
template <int Q, class S>
__global__ void k_bc_neq_all(const int32_t *list, const int8_t *setb, int64_t nl, int64_t n, const int32_t *nbr,
                             const typename Store<S>::C *rho, const typename Store<S>::C *u, S *f, BcVel ub,
                             double *tmp, int phase, int *err, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    const int b = setb[j];
    constexpr int W = Q == 19 ? 14 : 18;
    for (int t = 0; t < W; ++t) {
        const int k = Q == 19 ? c_bdry19[b][t] : c_bdry27[b][t];
        if (k < 0) break;
        if (phase == 0) {
            const int32_t nb = k == 0 ? (int32_t)i : nbr[(int64_t)(k - 1) * n + i];
            if (nb < 0) {
                atomicOr(err, DEVERR_MISSING_BC_NBR);
                tmp[t * nl + j] = (double)full_sh<S>(sh, T::ld(f, k * n + i), k);
                continue;
            }
            const C fw = feq_g<Q, C>(k, rho[i], (C)ub.u[b][0], (C)ub.u[b][1], (C)ub.u[b][2]);
            const C fn = feq_g<Q, C>(k, rho[nb], u[nb], u[n + nb], u[2 * n + nb]);
            tmp[t * nl + j] = (double)(fw + full_sh<S>(sh, T::ld(f, k * n + nb), k) - fn);
        } else {
            T::st(f, k * n + i, stored_sh<S>(sh, (C)tmp[t * nl + j], k));
        }
    }
}

// Restated inlet/outflow on the x faces: West wall cells hold
// fcol = feq(rho0, u_bc) (BC/ZouHe_Velocity.cpp:62-115 writes the
// equilibrium at the boundary cell's own, never-updated density), East wall
// cells copy the inner cell's fcol (BC/Outflow.cpp:39-52).
template <int Q, class S>
__global__ void k_bc_inout(const int32_t *list, int64_t nl, int east, int64_t n, const int32_t *nbr, double rho0,
                           S *f, S *fcol, double ubx, double uby, double ubz, int *err, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    const int32_t nb = nbr[(int64_t)((east ? 2 : 1) - 1) * n + i];
    if (nb < 0) {
        atomicOr(err, DEVERR_MISSING_BC_NBR);
        return;
    }
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        if (east) {
            const S v = fcol[k * n + nb];
            fcol[k * n + i] = v;
            f[k * n + i] = v;
        } else {
            const C v = stored_sh<S>(sh, feq_g<Q, C>(k, (C)rho0, (C)ubx, (C)uby, (C)ubz), k);
            T::st(fcol, k * n + i, v);
            T::st(f, k * n + i, v);
        }
    }
}

// Restated wet-node boundaries on the x faces (MT_BC_ZOUHE_HH, D3Q19):
// after the level-0 stream the West / East shell cells pull from their
// neighbours like fluid cells (a missing source keeps f) and complete the
// populations that come from outside the box -- West: the Zou-He velocity
// inlet with the Hecht-Harting transverse corrections (the formula family of
// BC/ZouHe_Velocity.cpp:81-93,170-199); East: the five incoming populations
// copied from the inner neighbour's streamed ones (BC/Outflow.cpp:39-52).
// The formulas are those of a textbook stream; under the reference's
// reversed pull they act on g_k = f_inv(k) with the velocity -u_bc.
// k_bc_wall_collide then collides the completed cells (LBGK, level-0 tau).
template <class S>
__global__ void k_bc_hh(const int32_t *list, int64_t nl, int east, int64_t n, int textbook,
                        const int32_t *__restrict__ nbr, const S *__restrict__ fcol, S *__restrict__ f, double ux,
                        double uy, double uz, int *err, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    C g[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) {
        const int m = textbook ? k : inv(k);
        const int32_t src = m == 0 ? (int32_t)i : nbr[(int64_t)((textbook ? inv(m) : m) - 1) * n + i];
        g[k] = full_sh<S>(sh, src >= 0 ? T::ld(fcol, (int64_t)m * n + src) : T::ld(f, (int64_t)m * n + i), m);
    }
    const C sgn = textbook ? C(1) : C(-1);
    if (!east) {
        const C Ux = sgn * (C)ux, Uy = sgn * (C)uy, Uz = sgn * (C)uz;
        const C rho = (g[0] + g[3] + g[4] + g[5] + g[6] + g[15] + g[16] + g[17] + g[18] +
                       C(2) * (g[2] + g[8] + g[10] + g[12] + g[14])) / (C(1) - Ux);
        const C ny = C(0.5) * (g[3] + g[15] + g[17] - g[4] - g[16] - g[18]) - rho * Uy / C(3);
        const C nz = C(0.5) * (g[5] + g[15] + g[18] - g[6] - g[16] - g[17]) - rho * Uz / C(3);
        g[1] = g[2] + rho * Ux / C(3);
        g[7] = g[8] + rho * (Ux + Uy) / C(6) - ny;
        g[9] = g[10] + rho * (Ux - Uy) / C(6) + ny;
        g[11] = g[12] + rho * (Ux + Uz) / C(6) - nz;
        g[13] = g[14] + rho * (Ux - Uz) / C(6) + nz;
    } else {
        const int32_t nb = nbr[(int64_t)(2 - 1) * n + i];  // the cell at -x
        if (nb < 0) {
            atomicOr(err, DEVERR_MISSING_BC_NBR);
            return;
        }
        const int in_e[5] = {2, 8, 10, 12, 14};
#pragma unroll
        for (int t = 0; t < 5; ++t) {
            const int k = in_e[t], m = textbook ? k : inv(k);
            g[k] = full_sh<S>(sh, T::ld(f, (int64_t)m * n + nb), m);
        }
    }
#pragma unroll
    for (int k = 0; k < 19; ++k) {
        const int m = textbook ? k : inv(k);
        T::st(f, (int64_t)m * n + i, stored_sh<S>(sh, g[k], m));
    }
}

template <class S>
__global__ void k_bc_wall_collide(const int32_t *list, int64_t nl, int64_t n, double tau, const S *__restrict__ f,
                                  S *__restrict__ fcol, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    C d[19];
#pragma unroll
    for (int k = 0; k < 19; ++k) d[k] = full_sh<S>(sh, T::ld(f, (int64_t)k * n + i), k);
    C r, x, y, z;
    macros_g<19, C>(d, r, x, y, z);
    collide_store<19, S, MT_COLL_LBGK>(d, r, x, y, z, tau, fcol, n, i, sh);
}

// D3Q19_BC_Strategy::initial_Feq (D3Q19_BC_Manager.hpp:157-167) on one
// boundary set: f = fcol = feq(rho0, u) with the face's velocity
template <int Q, class S>
__global__ void k_bc_set_eq(const int32_t *list, int64_t nl, int64_t n, double rho0, double ux, double uy, double uz,
                            S *f, S *fcol, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double v = feq_ref<Q>(k, rho0, ux, uy, uz);
        const C st = stored_f64<S>(sh, v, k);
        T::st(f, k * n + i, st);
        T::st(fcol, k * n + i, st);
    }
}

// SinglePointInterpolation::treat (ComplexBoundary_Manager.cpp:43-225) on
// one cell: wall links by Filippova-Haenel or distance-weighted
// interpolation, free links by plain pull, density clamp, eight
// multi-direct-forcing sweeps (each cell only touches its own populations:
// the sweeps run in registers).  g receives the new f, (fx, fy, fz) the
// cell's momentum-exchange force.
template <int Q, int FH, class S>
__device__ __forceinline__ void ib_cell(int64_t i, int64_t n, const double *dr, const int32_t *nbr, const S *fcol,
                                        typename Store<S>::C rho_b, typename Store<S>::C *g,
                                        typename Store<S>::C &fx, typename Store<S>::C &fy,
                                        typename Store<S>::C &fz, const Shift &sh)
{
    using T = Store<S>;
    using C = typename T::C;
    auto FC = [&](int k, int64_t idx) { return full_sh<S>(sh, T::ld(fcol, k * n + idx), k); };
    g[0] = FC(0, i);
    fx = 0;
    fy = 0;
    fz = 0;
#pragma unroll
    for (int k = 1; k < Q; ++k) {
        const C dd = (C)dr[inv(k) - 1];
        if (dr[inv(k) - 1] != -1.) {
            const C finc = FC(inv(k), i);
            const int32_t si = nbr[(int64_t)(inv(k) - 1) * n + i];
            const C fstr = si >= 0 ? FC(k, si) : finc;
            C fnew;
            if (FH) {
                if (dd < (C)0.5) {
                    fnew = ((C)1.0 - (C)2.0 * dd) * finc + (C)2.0 * dd * fstr;
                } else {
                    const C feqw = (C)w19z(inv(k)) * rho_b;
                    const C inv2d = (C)1.0 / ((C)2.0 * dd);
                    fnew = inv2d * fstr + ((C)1.0 - inv2d) * feqw;
                }
            } else {
                fnew = ((C)1.0 - dd) * finc + dd * fstr;
            }
            g[k] = fnew;
            const C mt = finc + fnew;
            fx += -mt * ex(k);
            fy += -mt * ey(k);
            fz += -mt * ez(k);
        } else {
            const int32_t si = nbr[(int64_t)(k - 1) * n + i];
            g[k] = si < 0 ? FC(inv(k), i) : FC(k, si);
        }
    }
    C ra = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) ra += g[k];
    if (ra < (C)0.3)
        g[0] += (C)1.0 * ((C)0.3 - ra);
    else if (ra < (C)0.5)
        g[0] += (C)0.5 * ((C)0.5 - ra);
    else if (ra > (C)3.0)
        g[0] += (C)1.0 * ((C)3.0 - ra);
    else if (ra > (C)2.0)
        g[0] += (C)0.5 * ((C)2.0 - ra);
    for (int it = 0; it < 8; ++it) {
        C r = 0, ux = 0, uy = 0, uz = 0;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            r += g[k];
            ux += g[k] * ex(k);
            uy += g[k] * ey(k);
            uz += g[k] * ez(k);
        }
        if (r <= (C)0.) continue;
        ux = ux / r;
        uy = uy / r;
        uz = uz / r;
        const C um = sqrt(ux * ux + uy * uy + uz * uz);
        if (um < (C)1e-10) continue;
        const C mx = (C)-0.5 * r * ux, my = (C)-0.5 * r * uy, mz = (C)-0.5 * r * uz;
        C adj = 0;
#pragma unroll
        for (int k = 1; k < Q; ++k) {
            if (dr[inv(k) - 1] == -1.) continue;
            const C df = (C)w19z(k) * (C)3.0 * (ex(k) * mx + ey(k) * my + ez(k) * mz);
            g[k] += df;
            adj -= df;
        }
        g[0] += adj;
    }
}

template <int Q, int FH, class S>
__global__ void k_ib_treat(const int32_t *list, int64_t nl, int64_t n, const int32_t *disrow, const double *dis,
                           const int32_t *nbr, const S *fcol, const typename Store<S>::C *rho, S *f, double *force, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    const double *dr = dis + (int64_t)disrow[i] * (Q - 1);
    C g[Q], fx, fy, fz;
    ib_cell<Q, FH, S>(i, n, dr, nbr, fcol, rho[i], g, fx, fy, fz, sh);
#pragma unroll
    for (int k = 0; k < Q; ++k) T::st(f, k * n + i, stored_sh<S>(sh, g[k], k));
    force[j] = (double)fx;
    force[nl + j] = (double)fy;
    force[2 * nl + j] = (double)fz;
}

// ---- fused schedule ---------------------------------------------------------
// The level keeps two post-collision buffers.  A substep streams from the
// current one (fcol) and, in the same pass, runs the next substep's
// calculateMacros + collide on the streamed f, writing fnext.  Between the
// stream of one substep and the collision of the next the reference touches a
// lat_f cell's f only through treat() (IB cells, fused below) and a C2F
// cell's fcol only through the copy fcol = f, so the lookahead collision sees
// the same f as the reference's and gives the same populations.

// gather of one cell's streamed populations from the source indices src[k]
// (k >= 1; -1 = no neighbour): every load is issued before any store (f and
// fcol are distinct buffers), so the Q - 1 gathers overlap.  A missing
// neighbour keeps f (read back from f, not written).
template <int Q, class S>
__device__ __forceinline__ void pull_src(int64_t i, int64_t n, const int32_t *src, const S *__restrict__ fcol,
                                         S *__restrict__ f, S *v)
{
    v[0] = fcol[i];
#pragma unroll
    for (int k = 1; k < Q; ++k) v[k] = src[k] >= 0 ? fcol[k * n + src[k]] : f[k * n + i];
    f[i] = v[0];
#pragma unroll
    for (int k = 1; k < Q; ++k)
        if (src[k] >= 0) f[k * n + i] = v[k];
}

// pull_src with 32-bit element offsets (Q * n < 2^32)
template <int Q, class S>
__device__ __forceinline__ void pull_src32(uint32_t i, uint32_t n, const int32_t *src, const S *__restrict__ fcol,
                                           S *__restrict__ f, S *v)
{
    v[0] = fcol[i];
#pragma unroll
    for (int k = 1; k < Q; ++k)
        v[k] = src[k] >= 0 ? fcol[(uint32_t)k * n + (uint32_t)src[k]] : f[(uint32_t)k * n + i];
    f[i] = v[0];
#pragma unroll
    for (int k = 1; k < Q; ++k)
        if (src[k] >= 0) f[(uint32_t)k * n + i] = v[k];
}

template <int Q, class S>
__device__ __forceinline__ void pull_cell(int64_t i, int64_t n, int textbook, const int32_t *__restrict__ nbr,
                                          const S *__restrict__ fcol, S *__restrict__ f, S *v)
{
    int32_t src[Q];
#pragma unroll
    for (int k = 1; k < Q; ++k) src[k] = __ldg(nbr + (int64_t)((textbook ? inv(k) : k) - 1) * n + i);
    pull_src<Q, S>(i, n, src, fcol, f, v);
}

// ABPatternPull::stream then the next collide, on lat_f cells that are not IB
// cells.
template <int Q, class S, int COLL>
__global__ void k_pull_collide(const int32_t *__restrict__ list, int64_t nl, int64_t n, int textbook,
                               const int32_t *__restrict__ nbr, const S *__restrict__ fcol, S *__restrict__ f,
                               S *__restrict__ fnext, double tau, typename Store<S>::C *__restrict__ rho,
                               typename Store<S>::C *__restrict__ u, int macros, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    C d[Q];
    {
        S v[Q];
        pull_cell<Q, S>(i, n, textbook, nbr, fcol, f, v);
#pragma unroll
        for (int k = 0; k < Q; ++k) d[k] = full_sh<S>(sh, T::cv(v[k]), k);
    }
    C r, x, y, z;
    macros_collide_store<Q, S, COLL>(d, r, x, y, z, tau, fnext, n, i, sh);
    if (macros) {
        rho[i] = r;
        u[i] = x;
        u[n + i] = y;
        u[2 * n + i] = z;
    }
}

// stream on overlap_C2F cells and their next collision, fcol = f
// (Collision_Manager.cpp:45-52)
template <int Q, class S>
__global__ void k_pull_copy(const int32_t *__restrict__ list, int64_t nl, int64_t n, int textbook,
                            const int32_t *__restrict__ nbr, const S *__restrict__ fcol, S *__restrict__ f,
                            S *__restrict__ fnext)
{
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    S v[Q];
    pull_cell<Q, S>(i, n, textbook, nbr, fcol, f, v);
#pragma unroll
    for (int k = 0; k < Q; ++k) fnext[k * n + i] = v[k];
}

// The fused pass over 4x4x4 bricks, one brick per warp (two cells per lane,
// local Morton index lane and lane + 32).  halo[216 * b + h] holds the cell
// index of position h = hx + 6 hy + 36 hz of the brick's 6x6x6 neighbourhood
// (local coordinates hx - 1, hy - 1, hz - 1; -1 = no cell), resolved once
// from the bricks' starts and occupancy masks; the warp stages it in shared
// memory, so a cell's Q - 1 source indices are shared-memory reads at fixed
// offsets.  The brick neighbours come from Morton_Assist::find_neighbor on a
// corner cell, so each source is the cell the reference's find() returns.
// Resident blocks per SM of each form and storage: brick_min_blocks.
// bcls: 1 stream + collide, 3 the same with the streamed f stored, 2 stream
// (f stored) + copy, 4 a direct-forcing band cell (stream; collided after
// the forcing).  The streamed f of class-1 cells is read by nothing in
// the coarse step (their next collision is computed here, a missing link's
// f never changes), so it is stored only when `fall` is set or when the
// state leaves the fused schedule (k_brick_pull).
// When `macros` is set (the level's last substep of the coarse step) the
// macros of the streamed f are written too: they are what the all-level
// calculateMacros at the end of the coarse step computes.

// The part of a brick cell's pass after its gather: v holds the streamed f
// of cell i (class cls), present(k) says whether link k had a source cell
// (a missing one keeps f, which is then not stored again).
template <int Q, class S, int COLL, class P>
__device__ __forceinline__ void brick_finish(uint32_t i, int cls, const S *v, P present, uint32_t n,
                                             S *__restrict__ f, S *__restrict__ fnext, double tau,
                                             typename Store<S>::C *__restrict__ rho,
                                             typename Store<S>::C *__restrict__ u, int macros, int fall,
                                             long long *__restrict__ acc, const Shift &sh)
{
    using T = Store<S>;
    using C = typename T::C;
    if (cls != 1 || fall) {
        f[i] = v[0];
#pragma unroll
        for (int k = 1; k < Q; ++k)
            if (present(k)) f[(uint32_t)k * n + i] = v[k];
    }
    if (cls == 2) {
#pragma unroll
        for (int k = 0; k < Q; ++k) fnext[(uint32_t)k * n + i] = v[k];
        return;
    }
    if (cls == 4) {
        // direct-forcing band: collided after the forcing; with acc the
        // band's rho, unforced velocity and cleared accumulator are
        // written here (what k_band_macros computes from the stored f)
        if constexpr (COLL == MT_COLL_LBGK) {
            if (acc) {
                C d[Q];
#pragma unroll
                for (int k = 0; k < Q; ++k) d[k] = full_sh<S>(sh, T::cv(v[k]), k);
                C r, x, y, z;
                macros_g<Q, C>(d, r, x, y, z);
                rho[i] = r;
                u[i] = x;
                u[n + i] = y;
                u[2 * n + i] = z;
                acc[i] = 0;
                acc[n + i] = 0;
                acc[2 * n + i] = 0;
            }
        }
        return;
    }
    C d[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) d[k] = full_sh<S>(sh, T::cv(v[k]), k);
    C r, x, y, z;
    macros_collide_store<Q, S, COLL>(d, r, x, y, z, tau, fnext, n, i, sh);
    if (macros) {
        rho[i] = r;
        u[i] = x;
        u[n + i] = y;
        u[2 * n + i] = z;
    }
}

// one cell (local Morton index m) of brick b in the fused brick pass
template <int Q, class S, int COLL>
__device__ __forceinline__ void brick_cell(int64_t b, int m, const int32_t *s_idx, const uint8_t *__restrict__ bcls,
                                           uint32_t n, int textbook, bool full, const S *__restrict__ fcol,
                                           S *__restrict__ f, S *__restrict__ fnext, double tau,
                                           typename Store<S>::C *__restrict__ rho,
                                           typename Store<S>::C *__restrict__ u, int macros, int fall,
                                           long long *__restrict__ acc, const Shift &sh)
{
    const int lx = (m & 1) | ((m >> 2) & 2), ly = ((m >> 1) & 1) | ((m >> 3) & 2),
              lz = ((m >> 2) & 1) | ((m >> 4) & 2);
    const int base = (lx + 1) + 6 * (ly + 1) + 36 * (lz + 1);
    const int32_t ii = s_idx[base];
    if (ii < 0) return;
    const int cls = __ldg(bcls + 64 * b + m);
    if (!cls) return;
    const uint32_t i = (uint32_t)ii;
    int32_t src[Q];
#pragma unroll
    for (int k = 1; k < Q; ++k) {
        const int off = ex(k) + 6 * ey(k) + 36 * ez(k);
        src[k] = s_idx[base + (textbook ? -off : off)];
    }
    S v[Q];
    v[0] = fcol[i];
    if (full) {
#pragma unroll
        for (int k = 1; k < Q; ++k) v[k] = fcol[(uint32_t)k * n + (uint32_t)src[k]];
    } else {
#pragma unroll
        for (int k = 1; k < Q; ++k)
            v[k] = src[k] >= 0 ? fcol[(uint32_t)k * n + (uint32_t)src[k]] : f[(uint32_t)k * n + i];
    }
    brick_finish<Q, S, COLL>(i, cls, v, [&](int k) { return full || src[k] >= 0; }, n, f, fnext, tau, rho, u,
                             macros, fall, acc, sh);
}

// one warp's brick b (see above); s_idx is the warp's 216-entry shared table;
// UNROLL (form 3): the lane's two cells in one unrolled sequence
template <int Q, class S, int COLL, bool UNROLL = false>
__device__ __forceinline__ void brick_warp(int64_t b, int lane, int32_t *s_idx, const int32_t *__restrict__ halo,
                                           const uint8_t *__restrict__ bcls, uint32_t n, int textbook,
                                           const S *__restrict__ fcol, S *__restrict__ f, S *__restrict__ fnext,
                                           double tau, typename Store<S>::C *__restrict__ rho,
                                           typename Store<S>::C *__restrict__ u, int macros, int fall,
                                           long long *__restrict__ acc, const Shift &sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int32_t *hb = halo + 216 * b;
    bool ok = true;
    for (int h = lane; h < 216; h += 32) {
        const int32_t e = __ldg(hb + h);
        s_idx[h] = e;
        ok &= e >= 0;
    }
    // every position of the neighbourhood holds a cell: no missing-link test per gather
    const bool full = __all_sync(0xffffffffu, ok);
    __syncwarp();
    if constexpr (UNROLL) {
        // both cells in one sequence: the second cell's gathers can be issued
        // before the first cell's collision
#pragma unroll
        for (int part = 0; part < 2; ++part)
            brick_cell<Q, S, COLL>(b, lane + 32 * part, s_idx, bcls, n, textbook, full, fcol, f, fnext, tau, rho, u,
                                   macros, fall, acc, sh);
    } else {
#pragma unroll 1
        for (int part = 0; part < 2; ++part)
            brick_cell<Q, S, COLL>(b, lane + 32 * part, s_idx, bcls, n, textbook, full, fcol, f, fnext, tau, rho, u,
                                   macros, fall, acc, sh);
    }
}

// The reduced-precision form of brick_warp: both cells of a lane are
// gathered first, then collided together with packed FP32 pairs (mt_pack2.cuh).
// Cells that stream without colliding (class 2), band cells (class 4) and
// absent cells take their own scalar paths; when only one cell of the pair
// collides, the other lane of the pair repeats its values and is not stored.
template <int Q, class S, int COLL>
__device__ __forceinline__ void brick_warp_pair(int64_t b, int lane, int32_t *s_idx, const int32_t *__restrict__ halo,
                                                const uint8_t *__restrict__ bcls, uint32_t n, int textbook,
                                                const S *__restrict__ fcol, S *__restrict__ f, S *__restrict__ fnext,
                                                double tau, float *__restrict__ rho, float *__restrict__ u, int macros,
                                                int fall, long long *__restrict__ acc, const Shift &sh)
{
    using T = Store<S>;
    const int32_t *hb = halo + 216 * b;
    for (int h = lane; h < 216; h += 32) s_idx[h] = __ldg(hb + h);
    __syncwarp();
    int base[2], cls[2];
    uint32_t idx[2];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const int m = lane + 32 * p;
        const int lx = (m & 1) | ((m >> 2) & 2), ly = ((m >> 1) & 1) | ((m >> 3) & 2),
                  lz = ((m >> 2) & 1) | ((m >> 4) & 2);
        base[p] = (lx + 1) + 6 * (ly + 1) + 36 * (lz + 1);
        const int32_t ii = s_idx[base[p]];
        cls[p] = ii >= 0 ? (int)__ldg(bcls + 64 * b + m) : 0;
        idx[p] = ii >= 0 ? (uint32_t)ii : 0u;
    }
    if (!cls[0] && !cls[1]) return;
    bool coll[2];
    float2 d[Q];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        coll[p] = cls[p] == 1 || cls[p] == 3;
        if (!cls[p]) continue;
        const uint32_t i = idx[p];
        const bool keep_f = cls[p] != 1 || fall;
        // gather, store what this cell's class stores, keep the full FP32 value
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            const int off = ex(k) + 6 * ey(k) + 36 * ez(k);
            const int32_t src = k ? s_idx[base[p] + (textbook ? -off : off)] : (int32_t)i;
            const S val = src >= 0 ? fcol[(uint32_t)k * n + (uint32_t)src] : f[(uint32_t)k * n + i];
            if (keep_f && src >= 0) f[(uint32_t)k * n + i] = val;
            if (cls[p] == 2) fnext[(uint32_t)k * n + i] = val;
            const float fv = full_sh<S>(sh, T::cv(val), k);
            if (p == 0)
                d[k].x = fv;
            else
                d[k].y = fv;
        }
        if constexpr (COLL == MT_COLL_LBGK) {
            if (cls[p] == 4 && acc) {
                // direct-forcing band: macros of the streamed f, accumulator cleared
                float dd[Q];
#pragma unroll
                for (int k = 0; k < Q; ++k) dd[k] = p == 0 ? d[k].x : d[k].y;
                float r, x, y, z;
                macros_g<Q, float>(dd, r, x, y, z);
                rho[i] = r;
                u[i] = x;
                u[n + i] = y;
                u[2 * n + i] = z;
                acc[i] = 0;
                acc[n + i] = 0;
                acc[2 * n + i] = 0;
            }
        }
    }
    if (!coll[0] && !coll[1]) return;
    // a pair with one colliding cell: the other lane repeats its values
    if (!coll[1]) {
#pragma unroll
        for (int k = 0; k < Q; ++k) d[k].y = d[k].x;
    } else if (!coll[0]) {
#pragma unroll
        for (int k = 0; k < Q; ++k) d[k].x = d[k].y;
    }
    float2 r, x, y, z;
    p2::macros<Q>(d, r, x, y, z);
    if (macros) {
        if (coll[0]) {
            rho[idx[0]] = r.x;
            u[idx[0]] = x.x;
            u[n + idx[0]] = y.x;
            u[2 * n + idx[0]] = z.x;
        }
        if (coll[1]) {
            rho[idx[1]] = r.y;
            u[idx[1]] = x.y;
            u[n + idx[1]] = y.y;
            u[2 * n + idx[1]] = z.y;
        }
    }
    float2 o[Q];
    if constexpr (COLL == MT_COLL_LBGK) {
        p2::lbgk<Q>(d, r, x, y, z, (float)(1.0 / tau), sh, o);  // stored deviations already
    } else {
        p2::cumulant(d, r, x, y, z, (float)(1.0 / tau), o);
#pragma unroll
        for (int k = 0; k < Q; ++k) o[k] = p2::sub(o[k], p2::bc(sh.v[k]));
    }
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        if (coll[0]) T::st(fnext, (uint32_t)k * n + idx[0], o[k].x);
        if (coll[1]) T::st(fnext, (uint32_t)k * n + idx[1], o[k].y);
    }
}

// brick_warp for every storage: V = 1 the pair form (reduced storages), V = 0
// the one-cell-at-a-time form
template <int Q, class S, int COLL, int V>
__device__ __forceinline__ void brick_warp_any(int64_t b, int lane, int32_t *s_idx, const int32_t *__restrict__ halo,
                                               const uint8_t *__restrict__ bcls, uint32_t n, int textbook,
                                               const S *__restrict__ fcol, S *__restrict__ f, S *__restrict__ fnext,
                                               double tau, typename Store<S>::C *__restrict__ rho,
                                               typename Store<S>::C *__restrict__ u, int macros, int fall,
                                               long long *__restrict__ acc, const Shift &sh)
{
    if constexpr (V == 1 && Store<S>::shifted && (COLL == MT_COLL_LBGK || Q == 27))
        brick_warp_pair<Q, S, COLL>(b, lane, s_idx, halo, bcls, n, textbook, fcol, f, fnext, tau, rho, u, macros,
                                    fall, acc, sh);
    else
        brick_warp<Q, S, COLL, V == 3>(b, lane, s_idx, halo, bcls, n, textbook, fcol, f, fnext, tau, rho, u, macros,
                                       fall, acc, sh);
}

#ifndef MT_BRICK_MIN_BLOCKS
#define MT_BRICK_MIN_BLOCKS 8  // resident 128-thread blocks per SM asked of the 16-bit one-cell passes (64 registers)
#endif
#ifndef MT_BRICK_MIN_BLOCKS_F32
#define MT_BRICK_MIN_BLOCKS_F32 7  // resident blocks asked of the FP32 one-cell passes (72 registers)
#endif
#ifndef MT_BRICK_MIN_BLOCKS_Q19_LBGK
#define MT_BRICK_MIN_BLOCKS_Q19_LBGK 10  // 16-bit D3Q19 LBGK one-cell passes: 48 registers, no spills
#endif
#ifndef MT_BRICK_PAIR_MIN_BLOCKS
#define MT_BRICK_PAIR_MIN_BLOCKS 4  // the pair passes of every reduced storage (128 registers)
#endif
// resident blocks per SM asked of a brick pass (V: one cell or a pair per step)
#ifndef MT_BRICK_WIDE_MIN_BLOCKS
#define MT_BRICK_WIDE_MIN_BLOCKS 6  // the one-cell form with more registers (85), reduced storages
#endif
#ifndef MT_BRICK_UNROLL_MIN_BLOCKS
#define MT_BRICK_UNROLL_MIN_BLOCKS 6  // the two cells of a lane in one unrolled sequence (form 3)
#endif
template <int Q, class S, int COLL, int V> constexpr int brick_min_blocks()
{
    if (V == 1 && Store<S>::shifted) return MT_BRICK_PAIR_MIN_BLOCKS;
    if (V == 2 && Store<S>::shifted) return MT_BRICK_WIDE_MIN_BLOCKS;
    if (V == 3) return Store<S>::shifted ? MT_BRICK_UNROLL_MIN_BLOCKS : 1;
    if (Store<S>::bytes == 2) return (COLL == MT_COLL_LBGK && Q == 19) ? MT_BRICK_MIN_BLOCKS_Q19_LBGK : MT_BRICK_MIN_BLOCKS;
    if (Store<S>::bytes == 4) return MT_BRICK_MIN_BLOCKS_F32;
    return 1;
}
// the form a level runs until mt_case_tune_bricks times them: form 0 for
// every storage (measured on the 4-level cumulant sphere and the
// direct-forcing sphere: the pair form runs 2-4x longer per launch at half
// the resident warps; FP32 form 0 at 7 resident blocks is as fast as or
// faster than forms 2 and 3 at 6)
template <class S> constexpr int brick_default_variant() { return 0; }

template <int Q, class S, int COLL, int V>
__global__ void __launch_bounds__(128, brick_min_blocks<Q, S, COLL, V>()) k_brick_step(
    int64_t nb, const int32_t *__restrict__ halo, const uint8_t *__restrict__ bcls, uint32_t n, int textbook,
    const S *__restrict__ fcol, S *__restrict__ f, S *__restrict__ fnext, double tau,
    typename Store<S>::C *__restrict__ rho, typename Store<S>::C *__restrict__ u, int macros, int fall,
    long long *__restrict__ acc, const Shift sh)
{
    __shared__ int32_t s_idx[4][216];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t b = 4 * (int64_t)blockIdx.x + w;
    if (b >= nb) return;
    brick_warp_any<Q, S, COLL, V>(b, lane, s_idx[w], halo, bcls, n, textbook, fcol, f, fnext, tau, rho, u, macros,
                                  fall, acc, sh);
}

// The same pass over the bricks of many cases (a batch): brick b of the work
// list belongs to the slot whose [off[s], off[s + 1]) range holds it; each
// slot carries one case level's tables, buffers and relaxation time.
template <int Q, class S, int COLL, int V>
__global__ void __launch_bounds__(128, brick_min_blocks<Q, S, COLL, V>()) k_brick_step_batch(const BrickBatch *__restrict__ bb,
                                                                                             const Shift sh)
{
    __shared__ int32_t s_idx[4][216];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t b = 4 * (int64_t)blockIdx.x + w;
    if (b >= bb->total) return;
    int lo = 0, hi = bb->nslots;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (bb->off[mid] <= b)
            lo = mid;
        else
            hi = mid;
    }
    const BrickSlot &sl = bb->slot[lo];
    using C = typename Store<S>::C;
    brick_warp_any<Q, S, COLL, V>(b - bb->off[lo], lane, s_idx[w], sl.halo, sl.cls, sl.n, sl.textbook,
                               (const S *)sl.fcol, (S *)sl.f, (S *)sl.fnext, sl.tau, (C *)sl.rho, (C *)sl.u, sl.macros,
                               sl.fall, sl.acc, sh);
}

// The streamed f of the class-1 cells, from the buffer the last fused pass
// read (the values that pass would have stored).
template <int Q, class S>
__global__ void __launch_bounds__(128) k_brick_pull(int64_t nb, const int32_t *__restrict__ halo,
                                                    const uint8_t *__restrict__ bcls, uint32_t n, int textbook,
                                                    const S *__restrict__ fcol, S *__restrict__ f)
{
    __shared__ int32_t s_idx[4][216];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t b = 4 * (int64_t)blockIdx.x + w;
    if (b >= nb) return;
    const int32_t *hb = halo + 216 * b;
    for (int h = lane; h < 216; h += 32) s_idx[w][h] = __ldg(hb + h);
    __syncwarp();
    for (int part = 0; part < 2; ++part) {
        const int m = lane + 32 * part;
        const int lx = (m & 1) | ((m >> 2) & 2), ly = ((m >> 1) & 1) | ((m >> 3) & 2),
                  lz = ((m >> 2) & 1) | ((m >> 4) & 2);
        const int base = (lx + 1) + 6 * (ly + 1) + 36 * (lz + 1);
        const int32_t ii = s_idx[w][base];
        if (ii < 0 || __ldg(bcls + 64 * b + m) != 1) continue;
        int32_t src[Q];
#pragma unroll
        for (int k = 1; k < Q; ++k) {
            const int off = ex(k) + 6 * ey(k) + 36 * ez(k);
            src[k] = s_idx[w][base + (textbook ? -off : off)];
        }
        S v[Q];
        pull_src32<Q, S>((uint32_t)ii, n, src, fcol, f, v);
    }
}

// treat() on the IB cells of the finest level, then their next collision.
// rho_b is the density calculateMacros(level) gives at the start of the
// substep: the macros of the cell's f before this treat.
template <int Q, int FH, class S, int COLL>
__global__ void k_ib_collide(const int32_t *list, int64_t nl, int64_t n, const int32_t *disrow, const double *dis,
                             const int32_t *nbr, const S *fcol, S *f, S *fnext, double tau, double *force,
                             typename Store<S>::C *rho, typename Store<S>::C *u, int macros, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nl) return;
    const int64_t i = list[j];
    const double *dr = dis + (int64_t)disrow[i] * (Q - 1);
    C g[Q], fx, fy, fz;
    {
#pragma unroll
        for (int k = 0; k < Q; ++k) g[k] = full_sh<S>(sh, T::ld(f, k * n + i), k);
        C r, x, y, z;
        macros_g<Q, C>(g, r, x, y, z);
        ib_cell<Q, FH, S>(i, n, dr, nbr, fcol, r, g, fx, fy, fz, sh);
    }
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const C st = stored_sh<S>(sh, g[k], k);
        T::st(f, k * n + i, st);
        // the next collision reads the stored value
        S sv;
        T::st(&sv, 0, st);
        g[k] = full_sh<S>(sh, T::cv(sv), k);
    }
    force[j] = (double)fx;
    force[nl + j] = (double)fy;
    force[2 * nl + j] = (double)fz;
    C r, x, y, z;
    macros_collide_store<Q, S, COLL>(g, r, x, y, z, tau, fnext, n, i, sh);
    if (macros) {
        rho[i] = r;
        u[i] = x;
        u[n + i] = y;
        u[2 * n + i] = z;
    }
}

// ---- direct-forcing immersed boundary (Lagrangian markers) --------------------
// No reference counterpart: a rigid sphere represented by surface markers on
// the finest level, explicit direct forcing (Uhlmann 2005) with the 3-point
// kernel of Roma, Peskin & Berger (1999) and Guo forcing in the collision.
// The Eulerian force of a substep is spread into int64 fixed point (2^-32),
// so the atomic sums are exact and independent of the order of arrival.
constexpr double kForceScale = 4294967296.0;  // 2^32
constexpr double kForceInv = 1.0 / 4294967296.0;

__host__ __device__ __forceinline__ double roma3(double r)
{
    r = fabs(r);
    if (r <= 0.5) return (1.0 + sqrt(1.0 - 3.0 * r * r)) / 3.0;
    if (r <= 1.5) {
        const double a = 1.0 - r;
        return (5.0 - 3.0 * r - sqrt(1.0 - 3.0 * a * a)) / 6.0;
    }
    return 0.0;
}

// rho and the unforced velocity of the band cells from their streamed f; the
// band's force accumulator restarts from zero
template <int Q, class S>
__global__ void k_band_macros(const int32_t *band, int64_t nb, int64_t n, const S *f, typename Store<S>::C *rho,
                              typename Store<S>::C *u, long long *acc, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nb) return;
    const int64_t i = band[j];
    C d[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) d[k] = full_sh<S>(sh, T::ld(f, k * n + i), k);
    C r, x, y, z;
    macros_g<Q, C>(d, r, x, y, z);
    rho[i] = r;
    u[i] = x;
    u[n + i] = y;
    u[2 * n + i] = z;
    acc[i] = 0;
    acc[n + i] = 0;
    acc[2 * n + i] = 0;
}

// one marker: interpolate rho and u at X(t), force F = 2 rho (U - u), spread
// F dv phi into the band cells; fk receives -F dv (the force on the body)
// grid[(x - lo) + dx ((y - lo) + dy (z - lo))] = index of band cell (x, y, z) or -1
static __global__ void k_band_grid(const int32_t *band, int64_t nb, const uint64_t *key, int64_t lx, int64_t ly,
                            int64_t lz, int64_t dx, int64_t dy, int64_t dz, int32_t *grid)
{
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nb) return;
    const int32_t i = band[j];
    const uint64_t k = key[i];
    const int64_t x = (int64_t)compact3(k) - lx, y = (int64_t)compact3(k >> 1) - ly, z = (int64_t)compact3(k >> 2) - lz;
    if (x < 0 || y < 0 || z < 0 || x >= dx || y >= dy || z >= dz) return;
    grid[x + dx * (y + dy * z)] = i;
}

template <class C>
__global__ void k_df_markers(int64_t nm, const double *ref, const double *dv, double cx, double cy, double cz,
                             const double *path, int64_t period, const long long *tstep, const int32_t *grid,
                             int64_t lx, int64_t ly, int64_t lz, int64_t dx, int64_t dy, int64_t dz, int64_t n,
                             const C *rho, const C *u, long long *acc, double *fk)
{
    const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (m >= nm) return;
    const int64_t ph = *tstep % period;
    const double *pp = path + 6 * ph;
    const double X = cx + pp[0] + ref[m], Y = cy + pp[1] + ref[nm + m], Z = cz + pp[2] + ref[2 * nm + m];
    const double ubx = pp[3], uby = pp[4], ubz = pp[5];
    const int64_t ix = (int64_t)floor(X), iy = (int64_t)floor(Y), iz = (int64_t)floor(Z);
    // the kernel's factors per axis (a stencil weight is wx wy wz, multiplied
    // in that order as the per-point evaluation does)
    double wx[3], wy[3], wz[3];
#pragma unroll
    for (int o = 0; o < 3; ++o) {
        wx[o] = roma3((double)(ix + o - 1) + 0.5 - X);
        wy[o] = roma3((double)(iy + o - 1) + 0.5 - Y);
        wz[o] = roma3((double)(iz + o - 1) + 0.5 - Z);
    }
    int32_t idx[27];
    double r = 0.0, vx = 0.0, vy = 0.0, vz = 0.0;
#pragma unroll
    for (int c = 0; c < 27; ++c) {
        const int ox = c % 3, oy = (c / 3) % 3, oz = c / 9;
        const double wv = wx[ox] * wy[oy] * wz[oz];
        // only band cells take force; they all lie in the grid's box
        const int64_t gx = ix + ox - 1 - lx, gy = iy + oy - 1 - ly, gz = iz + oz - 1 - lz;
        const int32_t i = (gx >= 0 && gy >= 0 && gz >= 0 && gx < dx && gy < dy && gz < dz)
                              ? __ldg(grid + gx + dx * (gy + dy * gz))
                              : -1;
        idx[c] = i;
        if (i >= 0) {
            r += wv * (double)rho[i];
            vx += wv * (double)u[i];
            vy += wv * (double)u[n + i];
            vz += wv * (double)u[2 * n + i];
        }
    }
    const double fx = 2.0 * r * (ubx - vx), fy = 2.0 * r * (uby - vy), fz = 2.0 * r * (ubz - vz);
    const double d = dv[m];
#pragma unroll
    for (int c = 0; c < 27; ++c) {
        const int32_t i = idx[c];
        if (i < 0) continue;
        const double s = wx[c % 3] * wy[(c / 3) % 3] * wz[c / 9] * d;
        atomicAdd((unsigned long long *)(acc + i), (unsigned long long)__double2ll_rn(fx * s * kForceScale));
        atomicAdd((unsigned long long *)(acc + n + i), (unsigned long long)__double2ll_rn(fy * s * kForceScale));
        atomicAdd((unsigned long long *)(acc + 2 * n + i), (unsigned long long)__double2ll_rn(fz * s * kForceScale));
    }
    fk[m] = -fx * d;
    fk[nm + m] = -fy * d;
    fk[2 * nm + m] = -fz * d;
}

// the body force of one forcing step: a fixed-order sum of the markers'
// forces into the accumulator (fx, fy, fz, count), then the substep count
static __global__ void __launch_bounds__(256) k_df_sum(const double *fk, int64_t nm, double *part, unsigned *done,
                                                        double *acc, long long *tstep)
{
    // body force: a fixed-order tree over each block of 256 markers, then the
    // last block to finish sums the partials in block order (deterministic)
    __shared__ double s[3][256];
    __shared__ bool last;
    const int t = threadIdx.x;
    const int64_t j = blockIdx.x * (int64_t)256 + t;
    for (int c = 0; c < 3; ++c) s[c][t] = j < nm ? fk[c * nm + j] : 0.0;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w)
            for (int c = 0; c < 3; ++c) s[c][t] += s[c][t + w];
        __syncthreads();
    }
    if (t == 0) {
        for (int c = 0; c < 3; ++c) part[3 * blockIdx.x + c] = s[c][0];
        __threadfence();
        last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double a[3] = {0., 0., 0.};
    for (int64_t b = t; b < gridDim.x; b += 256)
        for (int c = 0; c < 3; ++c) a[c] += __ldcg(part + 3 * b + c);
    for (int c = 0; c < 3; ++c) s[c][t] = a[c];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (t < w)
            for (int c = 0; c < 3; ++c) s[c][t] += s[c][t + w];
        __syncthreads();
    }
    if (t == 0) {
        for (int c = 0; c < 3; ++c) acc[c] += s[c][0];
        acc[3] += 1.0;
        *tstep += 1;
        *done = 0u;
    }
}

// LBGK collision with Guo forcing on the band cells: u = (j + g / 2) / rho,
// fcol = f - (f - feq(rho, u)) / tau + (1 - 1 / (2 tau)) w [3 (e - u) + 9 (e.u) e].g
// (the band's rho and unforced velocity are written by k_band_macros)
template <int Q, class S>
__global__ void k_band_collide(const int32_t *band, int64_t nb, int64_t n, double tau, const S *f,
                               const long long *acc, S *fcol, const Shift sh)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= nb) return;
    const int64_t i = band[j];
    if constexpr (T::shifted) {
        // reduced precision: the stored deviations s = f - s_k throughout
        // (the shift sums to 1 and its first moment is u_s), the forcing term
        // as 3 (e.g - u.g) + 9 (e.u)(e.g)
        float sd[Q];
        float rd = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            sd[k] = T::ld(f, k * n + i);
            rd += sd[k];
            jx += sd[k] * ex(k);
            jy += sd[k] * ey(k);
            jz += sd[k] * ez(k);
        }
        const float gx = (float)((double)acc[i] * kForceInv), gy = (float)((double)acc[n + i] * kForceInv),
                    gz = (float)((double)acc[2 * n + i] * kForceInv);
        const float r = 1.f + rd;
        jx += sh.u[0];
        jy += sh.u[1];
        jz += sh.u[2];
        const float rs = (r > -1e-6f && r < 1e-6f) ? ((r < 0.f) ? -1e-6f : 1e-6f) : r;
        const float ir = 1.f / rs;
        const float x = (jx + 0.5f * gx) * ir, y = (jy + 0.5f * gy) * ir, z = (jz + 0.5f * gz) * ir;
        const float om = (float)(1.0 / tau);
        const float fpre = 1.f - 0.5f * om;
        const float uu = 1.5f * (x * x + y * y + z * z);
        const float ug = x * gx + y * gy + z * gz;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            const float eu = ex(k) * x + ey(k) * y + ez(k) * z;
            const float eg = ex(k) * gx + ey(k) * gy + ez(k) * gz;
            const float wk = (float)w<Q>(k);
            const float dfeq = wk * ((r - 1.f) + r * (3.f * eu + 4.5f * eu * eu - uu)) - sh.dw[k];
            const float ge = 3.f * (eg - ug) + 9.f * eu * eg;
            T::st(fcol, k * n + i, fmaf(om, dfeq - sd[k], sd[k]) + fpre * wk * ge);
        }
        return;
    }
    C d[Q];
    C r = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        d[k] = full_sh<S>(sh, T::ld(f, k * n + i), k);
        r += d[k];
        jx += d[k] * ex(k);
        jy += d[k] * ey(k);
        jz += d[k] * ez(k);
    }
    // times 2^-32: exactly the division by the power-of-two scale
    const C gx = (C)((double)acc[i] * kForceInv), gy = (C)((double)acc[n + i] * kForceInv),
            gz = (C)((double)acc[2 * n + i] * kForceInv);
    const C rs = (r > C(-1e-6) && r < C(1e-6)) ? ((r < C(0)) ? C(-1e-6) : C(1e-6)) : r;
    const C x = (jx + gx * C(0.5)) / rs, y = (jy + gy * C(0.5)) / rs, z = (jz + gz * C(0.5)) / rs;
    const C om = C(1) / C(tau);
    const C fpre = C(1) - C(0.5) * om;
    const C uu = x * x + y * y + z * z;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const C eu = ex(k) * x + ey(k) * y + ez(k) * z;
        const C feq = r * (C)w<Q>(k) * (C(1) + C(3) * eu + C(4.5) * eu * eu - C(1.5) * uu);
        const C ge = (C(3) * (ex(k) - x) + C(9) * eu * ex(k)) * gx + (C(3) * (ey(k) - y) + C(9) * eu * ey(k)) * gy +
                     (C(3) * (ez(k) - z) + C(9) * eu * ez(k)) * gz;
        const C out = d[k] - (d[k] - feq) * om + fpre * (C)w<Q>(k) * ge;
        T::st(fcol, k * n + i, stored_sh<S>(sh, out, k));
    }
}

// fixed-order reduction of the per-cell IB force into the accumulator
// (LBM_Manager::accumIBForce, one call per treat): stage 1 sums 256-cell
// chunks into partials, stage 2 sums the partials in order
static __global__ void k_force_partial(const double *force, int64_t nl, double *partial)
{
    __shared__ double s[3][256];
    const int t = threadIdx.x;
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + t;
    for (int c = 0; c < 3; ++c) s[c][t] = j < nl ? force[c * nl + j] : 0.0;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (t < w)
            for (int c = 0; c < 3; ++c) s[c][t] += s[c][t + w];
        __syncthreads();
    }
    if (t == 0)
        for (int c = 0; c < 3; ++c) partial[c * gridDim.x + blockIdx.x] = s[c][0];
}

static __global__ void k_force_reduce(const double *force, int64_t nl, double *acc)
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

static __global__ void k_force_tick(double *acc) { acc[3] += 1.0; }

template <int Q, class S>
__global__ void k_to_f64(const S *src, double *dst, int64_t n, const Shift sh)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int k = 0; k < Q; ++k) dst[k * n + i] = (double)full_sh<S>(sh, Store<S>::ld(src, k * n + i), k);
}
template <int Q, class S>
__global__ void k_from_f64(const double *src, S *dst, int64_t n, const Shift sh)
{
    using C = typename Store<S>::C;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        const double v = src[k * n + i];
        Store<S>::st(dst, k * n + i, stored_f64<S>(sh, v, k));
    }
}
template <class C>
__global__ void k_macro_to_f64(const C *src, double *dst, int64_t m)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < m) dst[i] = (double)src[i];
}
template <class S>
__global__ void k_guard(const S *f, const S *fcol, int64_t total, int *err)
{
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    bool bad = false;
    for (; j < total; j += (int64_t)gridDim.x * blockDim.x)
        bad |= !isfinite((double)Store<S>::ld(f, j)) || !isfinite((double)Store<S>::ld(fcol, j));
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, DEVERR_NONFINITE);
}

// ----------------------------------------------------------------------------
// host side
// ----------------------------------------------------------------------------
template <class S> struct AmrTyped {
    using C = typename Store<S>::C;
    static S *f(Level &lv) { return (S *)lv.f; }
    static S *fcol(Level &lv) { return (S *)lv.fcol; }
    static C *rho(Level &lv) { return (C *)lv.rho; }
    static C *u(Level &lv) { return (C *)lv.u; }
};

inline int upload_bdry_tables(Ctx &ctx)
{
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
    return MT_OK;
}

// boundary sets of each face strategy (West, East, South, North, Bot, Top):
// the face, its edges and corners as NonEquilibrumExtrapolation.hpp:24-110
// registers them
static const int kFaceSets[6][9] = {
    {0, 7, 8, 15, 17, 19, 20, 23, 24}, {1, 6, 9, 14, 16, 18, 21, 22, 25},
    {2, 11, 13, -1, -1, -1, -1, -1, -1}, {3, 10, 12, -1, -1, -1, -1, -1, -1},
    {4, -1, -1, -1, -1, -1, -1, -1, -1}, {5, -1, -1, -1, -1, -1, -1, -1, -1}};

// Rescaling of the non-equilibrium part across a level interface.  The
// reference's factors (LBM_Manager.cpp:1065, 1137): 2 tau_f / tau_c onto the
// fine post-collision populations and tau_c / (2 tau_f) onto the coarse
// post-stream ones.  MT_SCALE_STANDARD uses the rescaling that keeps the
// physical viscous stress continuous under 2:1 convective scaling (Dupuis &
// Chopard 2003): fneq_f = tau_f / (2 tau_c) fneq_c, written for post-collision
// populations as (tau_f - 1) / (2 (tau_c - 1)), and fneq_c = 2 tau_c / tau_f fneq_f.
inline double c2f_scale(const Case &c, int fine)
{
    const double tf = c.d.tau[fine], tc = c.d.tau[fine - 1];
    return c.scaling == MT_SCALE_STANDARD ? (tf - 1.0) / (2.0 * (tc - 1.0)) : (2.0 * tf) / tc;
}
inline double f2c_scale(const Case &c, int coarse)
{
    const double tc = c.d.tau[coarse], tf = c.d.tau[coarse + 1];
    return c.scaling == MT_SCALE_STANDARD ? (2.0 * tc) / tf : tc / (2.0 * tf);
}

// the direct-forcing step on level l (after its stream): band macros, the
// markers' interpolation and spreading, the body force
// (band_macros_done: the level's brick pass already wrote the band macros)
template <class S, int Q>
int df_force(Ctx &ctx, Case &c, int l, bool band_macros_done = false)
{
    using A = AmrTyped<S>;
    using C = typename Store<S>::C;
    cudaStream_t s = ctx.stream;
    Level &lv = c.lv[l];
    if (!lv.nband) return MT_OK;
    if (!band_macros_done) {
        k_band_macros<Q, S><<<grid_for(lv.nband, 128), 128, 0, s>>>(lv.band, lv.nband, lv.n, A::f(lv), A::rho(lv),
                                                                     A::u(lv), c.acc, c.shift[l]);
        MT_LAUNCHED(ctx);
    }
    if (!c.nm) {
        k_force_tick<<<1, 1, 0, s>>>(c.force_acc);
        MT_LAUNCHED(ctx);
        return MT_OK;
    }
    k_df_markers<C><<<grid_for(c.nm, 64), 64, 0, s>>>(
        c.nm, c.mref, c.mdv, c.center[0], c.center[1], c.center[2], c.path, c.period, c.tstep, c.mgrid, c.mlo[0],
        c.mlo[1], c.mlo[2], c.mdim[0], c.mdim[1], c.mdim[2], lv.n, (const C *)A::rho(lv), (const C *)A::u(lv), c.acc,
        c.mforce);
    MT_LAUNCHED(ctx);
    const int64_t nbf = (c.nm + 255) / 256;
    k_df_sum<<<(unsigned)nbf, 256, 0, s>>>(c.mforce, c.nm, c.mforce + 3 * c.nm,
                                           (unsigned *)(c.mforce + 3 * (c.nm + nbf)), c.force_acc, c.tstep);
    MT_LAUNCHED(ctx);
    return MT_OK;
}

template <class S, int Q>
int band_collide(Ctx &ctx, Case &c, int l, void *out)
{
    using A = AmrTyped<S>;
    Level &lv = c.lv[l];
    if (!lv.nband) return MT_OK;
    k_band_collide<Q, S><<<grid_for(lv.nband, 64), 64, 0, ctx.stream>>>(lv.band, lv.nband, lv.n, c.d.tau[l],
                                                                         A::f(lv), c.acc, (S *)out, c.shift[l]);
    MT_LAUNCHED(ctx);
    return MT_OK;
}

// One fused brick pass of level l in the form `variant` (0 one cell per lane
// step; 3 the lane's two cells in one unrolled sequence; for the reduced
// storages also 1, a packed pair, and 2, one cell with more registers per
// thread) on stream s, writing the next collision into fnext.
template <int Q, class S>
void brick_launch(Case &c, int l, int variant, cudaStream_t s, S *fnext, int mac, int fall, long long *bacc)
{
    using A = AmrTyped<S>;
    Level &lv = c.lv[l];
    const unsigned g = grid_for(lv.nbrick, 4);
    const uint32_t n32 = (uint32_t)lv.n;
    const int tb = c.d.stream_convention;
    auto go = [&](auto coll, auto v) {
        constexpr int COLL = decltype(coll)::value, V = decltype(v)::value;
        k_brick_step<Q, S, COLL, V><<<g, 128, 0, s>>>(lv.nbrick, lv.bhalo, lv.bcls, n32, tb, A::fcol(lv), A::f(lv),
                                                      fnext, c.d.tau[l], A::rho(lv), A::u(lv), mac, fall,
                                                      COLL == MT_COLL_LBGK ? bacc : nullptr, c.shift[l]);
    };
    using LB = std::integral_constant<int, MT_COLL_LBGK>;
    using CU = std::integral_constant<int, MT_COLL_CUMULANT>;
    using V0 = std::integral_constant<int, 0>;
    using V1 = std::integral_constant<int, 1>;
    using V2 = std::integral_constant<int, 2>;
    using V3 = std::integral_constant<int, 3>;
    const int v = (Store<S>::shifted || variant == 3) ? variant : 0;
    if (c.d.collision == MT_COLL_LBGK) {
        if (v == 1) go(LB{}, V1{}); else if (v == 2) go(LB{}, V2{}); else if (v == 3) go(LB{}, V3{}); else go(LB{}, V0{});
    } else {
        if constexpr (Q == 27) {
            if (v == 1) go(CU{}, V1{}); else if (v == 2) go(CU{}, V2{}); else if (v == 3) go(CU{}, V3{}); else go(CU{}, V0{});
        }
    }
}

template <class S, int Q>
int amr_phase_q(Ctx &ctx, Case &c, int phase, int l)
{
    using A = AmrTyped<S>;
    const int B = 128;
    cudaStream_t s = ctx.stream;
    Level &lv = c.lv[l];
    const int64_t n = lv.n;
    switch (phase) {
    case PH_MACROS:
        if (lv.ncollide) {
            k_macros<Q, S><<<grid_for(lv.ncollide, B), B, 0, s>>>(lv.collide_list, lv.ncollide, n, A::f(lv),
                                                                   A::rho(lv), A::u(lv), c.shift[l]);
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    case PH_COLLIDE: {
        // the direct-forcing band collides with its force (band_collide)
        const int32_t *cl = lv.nband ? lv.collide_nb : lv.collide_list;
        const int64_t ncl = lv.nband ? lv.ncollide_nb : lv.ncollide;
        if (ncl) {
            if (c.d.collision == MT_COLL_LBGK) {
                k_collide<Q, S, MT_COLL_LBGK><<<grid_for(ncl, B), B, 0, s>>>(cl, ncl, n, c.d.tau[l], A::f(lv),
                                                                             A::rho(lv), A::u(lv), A::fcol(lv), c.shift[l]);
            } else {
                // the cumulant model exists for D3Q27 only (checked at case creation)
                if constexpr (Q == 27)
                    k_collide<Q, S, MT_COLL_CUMULANT><<<grid_for(ncl, 64), 64, 0, s>>>(
                        cl, ncl, n, c.d.tau[l], A::f(lv), A::rho(lv), A::u(lv), A::fcol(lv), c.shift[l]);
            }
            MT_LAUNCHED(ctx);
        }
        if (int rc = band_collide<S, Q>(ctx, c, l, A::fcol(lv))) return rc;
        if (lv.nlist[2]) {
            k_copy_fcol<Q, S><<<grid_for(lv.nlist[2], B), B, 0, s>>>(lv.list[2], lv.nlist[2], n, A::f(lv),
                                                                      A::fcol(lv));
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    }
    case PH_STREAM:
        if (lv.nstream) {
            k_stream<Q, S><<<grid_for(lv.nstream, B), B, 0, s>>>(lv.stream_list, lv.nstream, n, c.d.stream_convention,
                                                                  lv.nbr, A::fcol(lv), A::f(lv));
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    case PH_EXPLOSION:
    case PH_EXPLOSION_B: {
        // PH_EXPLOSION_B: the second substep's explosion of MT_ITIME_HOLD /
        // MT_ITIME_EXTRAP (the latter from the extrapolated parent state, then
        // the sources' values are kept for the next one)
        if (l < 1 || !lv.nexpl) return MT_OK;
        Level &cl = c.lv[l - 1];
        const double scale = c2f_scale(c, l);
        const bool ex = phase == PH_EXPLOSION_B && c.itime == MT_ITIME_EXTRAP;
        if (ex && !lv.expl_prev) return set_err(ctx, MT_ERR_STATE, "extrapolated explosion without saved sources");
        k_explosion<Q, S><<<grid_for(8 * lv.nexpl, B), B, 0, s>>>(lv.expl_src, lv.expl_child, lv.nexpl, cl.n, A::fcol(cl),
                                                               n, A::fcol(lv), scale, (S *)lv.fcol_alt,
                                                               lv.nexpl_f2c, c.shift[l - 1], c.shift[l],
                                                               ex ? (const S *)lv.expl_prev : nullptr);
        MT_LAUNCHED(ctx);
        if (ex) {
            k_expl_save<Q, S><<<grid_for(lv.nexpl, B), B, 0, s>>>(lv.expl_src, lv.nexpl, A::fcol(cl), cl.n,
                                                                (S *)lv.expl_prev);
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    }
    case PH_EXPL_SAVE: {
        // the sources' current parent values (the state was set or the option turned on)
        if (l < 1 || !lv.nexpl || !lv.expl_prev) return MT_OK;
        Level &cl = c.lv[l - 1];
        k_expl_save<Q, S><<<grid_for(lv.nexpl, B), B, 0, s>>>(lv.expl_src, lv.nexpl, A::fcol(cl), cl.n,
                                                            (S *)lv.expl_prev);
        MT_LAUNCHED(ctx);
        return MT_OK;
    }
    case PH_COALESCENCE: {
        if (l >= c.d.max_level || !lv.nlist[1]) return MT_OK;
        Level &fl = c.lv[l + 1];
        const double scale = f2c_scale(c, l);
        k_coalescence<Q, S><<<grid_for(lv.nlist[1], B), B, 0, s>>>(lv.list[1], lv.coal_child, lv.nlist[1], n,
                                                                    A::f(lv), A::f(fl), fl.n, scale, c.shift[l], c.shift[l + 1]);
        MT_LAUNCHED(ctx);
        return MT_OK;
    }
    case PH_BC:
    case PH_BC_FACE0 + 0: case PH_BC_FACE0 + 1: case PH_BC_FACE0 + 2:
    case PH_BC_FACE0 + 3: case PH_BC_FACE0 + 4: case PH_BC_FACE0 + 5: {
        // all six face groups in the reference's order (LBM_Simulator.cpp:90-95), or one
        const int f0 = phase == PH_BC ? 0 : phase - PH_BC_FACE0, f1 = phase == PH_BC ? 6 : f0 + 1;
        Level &l0 = c.lv[0];
        if (phase == PH_BC && c.bc_all && c.nbc_all) {
            BcVel ub;
            for (int face = 0; face < 6; ++face)
                for (int g = 0; g < 9; ++g) {
                    const int b = kFaceSets[face][g];
                    if (b < 0) break;
                    for (int a = 0; a < 3; ++a) ub.u[b][a] = c.face_u[face][a];
                }
            for (int ph = 0; ph < 2; ++ph) {
                k_bc_neq_all<Q, S><<<grid_for(c.nbc_all, B), B, 0, s>>>(c.bc_all, c.bc_setb, c.nbc_all, l0.n, l0.nbr,
                                                                         A::rho(l0), A::u(l0), A::f(l0), ub,
                                                                         c.bc_tmp_all, ph, c.dev_err, c.shift[0]);
                MT_LAUNCHED(ctx);
            }
            return MT_OK;
        }
        double *tmp = c.bc_tmp;
        if (!tmp) return MT_OK;
        for (int face = f0; face < f1; ++face)
            for (int g = 0; g < 9; ++g) {
                const int b = kFaceSets[face][g];
                if (b < 0) break;
                if (!l0.nbc[b]) continue;
                for (int ph = 0; ph < 2; ++ph) {
                    k_bc_neq<Q, S><<<grid_for(l0.nbc[b], B), B, 0, s>>>(
                        l0.bclist[b], l0.nbc[b], b, l0.n, l0.nbr, A::rho(l0), A::u(l0), A::f(l0), c.face_u[face][0],
                        c.face_u[face][1], c.face_u[face][2], tmp, ph, c.dev_err, c.shift[0]);
                    MT_LAUNCHED(ctx);
                }
            }
        return MT_OK;
    }
    case PH_BC_HH: {
        if constexpr (Q == 19) {
            Level &l0 = c.lv[0];
            for (int face = 0; face < 2; ++face) {
                if (!l0.nbc[face]) continue;
                k_bc_hh<S><<<grid_for(l0.nbc[face], B), B, 0, s>>>(l0.bclist[face], l0.nbc[face], face, l0.n,
                                                                    c.d.stream_convention, l0.nbr, A::fcol(l0),
                                                                    A::f(l0), c.face_u[0][0], c.face_u[0][1],
                                                                    c.face_u[0][2], c.dev_err, c.shift[0]);
                MT_LAUNCHED(ctx);
            }
            for (int face = 0; face < 2; ++face) {
                if (!l0.nbc[face]) continue;
                k_bc_wall_collide<S><<<grid_for(l0.nbc[face], B), B, 0, s>>>(l0.bclist[face], l0.nbc[face], l0.n,
                                                                              c.d.tau[0], A::f(l0), A::fcol(l0),
                                                                              c.shift[0]);
                MT_LAUNCHED(ctx);
            }
            return MT_OK;
        } else {
            return set_err(ctx, MT_ERR_ARG, "the Zou-He / Hecht-Harting boundary is D3Q19");
        }
    }
    case PH_BC_INOUT: {
        Level &l0 = c.lv[0];
        for (int face = 0; face < 2; ++face) {
            if (!l0.nbc[face]) continue;
            k_bc_inout<Q, S><<<grid_for(l0.nbc[face], B), B, 0, s>>>(l0.bclist[face], l0.nbc[face], face, l0.n, l0.nbr,
                                                                      c.d.rho0, A::f(l0), A::fcol(l0), c.face_u[0][0],
                                                                      c.face_u[0][1], c.face_u[0][2], c.dev_err, c.shift[0]);
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    }
    case PH_IB: {
        if (c.d.ib_method == MT_IB_DF) return df_force<S, Q>(ctx, c, c.d.max_level);
        Level &fl = c.lv[c.d.max_level];
        if (!fl.nib) {
            k_force_tick<<<1, 1, 0, s>>>(c.force_acc);
            MT_LAUNCHED(ctx);
            return MT_OK;
        }
        if (c.d.ib_method == MT_IB_FH)
            k_ib_treat<Q, 1, S><<<grid_for(fl.nib, 64), 64, 0, s>>>(fl.iblist, fl.nib, fl.n, fl.disrow, c.dis, fl.nbr,
                                                                     A::fcol(fl), A::rho(fl), A::f(fl), c.ib_force, c.shift[c.d.max_level]);
        else
            k_ib_treat<Q, 0, S><<<grid_for(fl.nib, 64), 64, 0, s>>>(fl.iblist, fl.nib, fl.n, fl.disrow, c.dis, fl.nbr,
                                                                     A::fcol(fl), A::rho(fl), A::f(fl), c.ib_force, c.shift[c.d.max_level]);
        MT_LAUNCHED(ctx);
        // ib_force holds 3 * nib per-cell values followed by room for the partials
        const unsigned nb = grid_for(fl.nib, 256);
        double *partial = c.ib_force + 3 * fl.nib;
        k_force_partial<<<nb, 256, 0, s>>>(c.ib_force, fl.nib, partial);
        MT_LAUNCHED(ctx);
        k_force_reduce<<<1, 256, 0, s>>>(partial, nb, c.force_acc);
        MT_LAUNCHED(ctx);
        return MT_OK;
    }
    case PH_F2C_COLLIDE:
        // the F2C share of collide(level) in the fused schedule: their f comes from coalescence
        if (lv.nlist[1]) {
            if (c.d.collision == MT_COLL_LBGK) {
                k_collide<Q, S, MT_COLL_LBGK><<<grid_for(lv.nlist[1], B), B, 0, s>>>(
                    lv.list[1], lv.nlist[1], n, c.d.tau[l], A::f(lv), A::rho(lv), A::u(lv), A::fcol(lv), c.shift[l]);
            } else {
                if constexpr (Q == 27)
                    k_collide<Q, S, MT_COLL_CUMULANT><<<grid_for(lv.nlist[1], 64), 64, 0, s>>>(
                        lv.list[1], lv.nlist[1], n, c.d.tau[l], A::f(lv), A::rho(lv), A::u(lv), A::fcol(lv), c.shift[l]);
            }
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    case PH_COAL_COLLIDE: {
        if (l >= c.d.max_level || !lv.nlist[1]) return MT_OK;
        Level &fl = c.lv[l + 1];
        const double scale = f2c_scale(c, l);
        if (c.d.collision == MT_COLL_LBGK) {
            k_coal_collide<Q, S, MT_COLL_LBGK><<<grid_for(lv.nlist[1], 64), 64, 0, s>>>(
                lv.list[1], lv.coal_child, lv.nlist[1], n, A::f(lv), A::f(fl), fl.n, scale, c.d.tau[l],
                (S *)lv.fcol_alt, A::rho(lv), A::u(lv), c.macros_now, c.shift[l], c.shift[l + 1]);
        } else {
            if constexpr (Q == 27)
                k_coal_collide<Q, S, MT_COLL_CUMULANT><<<grid_for(lv.nlist[1], 64), 64, 0, s>>>(
                    lv.list[1], lv.coal_child, lv.nlist[1], n, A::f(lv), A::f(fl), fl.n, scale, c.d.tau[l],
                    (S *)lv.fcol_alt, A::rho(lv), A::u(lv), c.macros_now, c.shift[l], c.shift[l + 1]);
        }
        MT_LAUNCHED(ctx);
        return MT_OK;
    }
    case PH_FACE_EQ0 + 0: case PH_FACE_EQ0 + 1: case PH_FACE_EQ0 + 2:
    case PH_FACE_EQ0 + 3: case PH_FACE_EQ0 + 4: case PH_FACE_EQ0 + 5: {
        const int face = phase - PH_FACE_EQ0;
        Level &l0 = c.lv[0];
        for (int g = 0; g < 9; ++g) {
            const int b = kFaceSets[face][g];
            if (b < 0) break;
            if (!l0.nbc[b]) continue;
            k_bc_set_eq<Q, S><<<grid_for(l0.nbc[b], B), B, 0, s>>>(l0.bclist[b], l0.nbc[b], l0.n, c.d.rho0,
                                                                    c.face_u[face][0], c.face_u[face][1],
                                                                    c.face_u[face][2], A::f(l0), A::fcol(l0), c.shift[0]);
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    }
    case PH_DF: {
        // after PH_PULL_COLLIDE: a brick level's pass (alone or batched) wrote the band macros
        if (int rc = df_force<S, Q>(ctx, c, l, lv.bricks)) return rc;
        return band_collide<S, Q>(ctx, c, l, lv.fcol_alt);
    }
    case PH_BAND_GRID:
        if (lv.nband && c.mgrid) {
            k_band_grid<<<grid_for(lv.nband, 256), 256, 0, s>>>(lv.band, lv.nband, lv.key, c.mlo[0], c.mlo[1], c.mlo[2],
                                                                c.mdim[0], c.mdim[1], c.mdim[2], c.mgrid);
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    case PH_SYNC_F:
        if (lv.bricks) {
            k_brick_pull<Q, S><<<grid_for(lv.nbrick, 4), 128, 0, s>>>(lv.nbrick, lv.bhalo, lv.bcls, (uint32_t)n,
                                                                       c.d.stream_convention, A::fcol(lv), A::f(lv));
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    case PH_PRIME:
        // lookahead of the fused schedule from the current f: the second
        // buffer gets every cell's fcol, then the collision of lat_f and F2C
        // and the copy of C2F (the first collide(level) of the next substep)
        if (!n) return MT_OK;
        MT_CUDA(ctx, cudaMemcpyAsync(lv.fcol_alt, lv.fcol, sizeof(S) * Q * n, cudaMemcpyDeviceToDevice, s));
        {
            const int32_t *cl = lv.nband ? lv.collide_nb : lv.collide_list;
            const int64_t ncl = lv.nband ? lv.ncollide_nb : lv.ncollide;
            if (ncl) {
                if (c.d.collision == MT_COLL_LBGK) {
                    k_collide<Q, S, MT_COLL_LBGK><<<grid_for(ncl, B), B, 0, s>>>(
                        cl, ncl, n, c.d.tau[l], A::f(lv), A::rho(lv), A::u(lv), (S *)lv.fcol_alt, c.shift[l]);
                } else {
                    if constexpr (Q == 27)
                        k_collide<Q, S, MT_COLL_CUMULANT><<<grid_for(ncl, 64), 64, 0, s>>>(
                            cl, ncl, n, c.d.tau[l], A::f(lv), A::rho(lv), A::u(lv), (S *)lv.fcol_alt, c.shift[l]);
                }
                MT_LAUNCHED(ctx);
            }
            if (int rc = band_collide<S, Q>(ctx, c, l, lv.fcol_alt)) return rc;
        }
        if (lv.nlist[2]) {
            k_copy_fcol<Q, S><<<grid_for(lv.nlist[2], B), B, 0, s>>>(lv.list[2], lv.nlist[2], n, A::f(lv),
                                                                      (S *)lv.fcol_alt);
            MT_LAUNCHED(ctx);
        }
        return MT_OK;
    case PH_PULL_COLLIDE: {
        // stream(level) of this substep fused with collide(level) of the next,
        // reading fcol and writing f and fcol_alt; treat() on the finest level
        // (its cells are disjoint from the fused pass: on the side stream when
        // the case has one, overlapping the pass)
        const int L = c.d.max_level;
        const bool ib_level = l == L && l > 0 && c.d.ib_method != MT_IB_DF;
        const int tb = c.d.stream_convention;
        const int mac = c.macros_now;
        // level 0's boundary sweep reads the streamed f of inner cells
        const int fall = (l == 0 && c.d.bc_mode == MT_BC_NEQ) ? 1 : 0;
        cudaStream_t is = s;
        if (ib_level && lv.nib && c.side && !c.no_side) {
            MT_CUDA(ctx, cudaEventRecord(c.ev_fork, s));
            MT_CUDA(ctx, cudaStreamWaitEvent(c.side, c.ev_fork, 0));
            is = c.side;
        }
        if (ib_level) {
            if (!lv.nib) {
                k_force_tick<<<1, 1, 0, s>>>(c.force_acc);
                MT_LAUNCHED(ctx);
            } else {
                const double tau = c.d.tau[l];
                auto ib = [&](auto fh, auto coll) {
                    constexpr int FH = decltype(fh)::value, COLL = decltype(coll)::value;
                    k_ib_collide<Q, FH, S, COLL><<<grid_for(lv.nib, 64), 64, 0, is>>>(
                        lv.iblist, lv.nib, n, lv.disrow, c.dis, lv.nbr, A::fcol(lv), A::f(lv), (S *)lv.fcol_alt, tau,
                        c.ib_force, A::rho(lv), A::u(lv), mac, c.shift[l]);
                };
                using I0 = std::integral_constant<int, 0>;
                using I1 = std::integral_constant<int, 1>;
                using LB = std::integral_constant<int, MT_COLL_LBGK>;
                using CU = std::integral_constant<int, MT_COLL_CUMULANT>;
                if (c.d.collision == MT_COLL_LBGK) {
                    if (c.d.ib_method == MT_IB_FH) ib(I1{}, LB{}); else ib(I0{}, LB{});
                } else {
                    if constexpr (Q == 27) {
                        if (c.d.ib_method == MT_IB_FH) ib(I1{}, CU{}); else ib(I0{}, CU{});
                    }
                }
                MT_LAUNCHED(ctx);
                const unsigned nb = grid_for(lv.nib, 256);
                double *partial = c.ib_force + 3 * lv.nib;
                k_force_partial<<<nb, 256, 0, is>>>(c.ib_force, lv.nib, partial);
                MT_LAUNCHED(ctx);
                k_force_reduce<<<1, 256, 0, is>>>(partial, nb, c.force_acc);
                MT_LAUNCHED(ctx);
            }
        }
        if (c.pull_mode == 1) {
            // the batch runs this level's bricks
        } else if (lv.bricks) {
            // the band's macros come out of the pass (the direct-forcing step skips k_band_macros)
            long long *bacc = (l == L && lv.nband) ? c.acc : nullptr;
            brick_launch<Q, S>(c, l, lv.brick_variant, s, (S *)lv.fcol_alt, mac, fall, bacc);
            MT_LAUNCHED(ctx);
        } else {
            if (lv.nfused) {
                if (c.d.collision == MT_COLL_LBGK) {
                    k_pull_collide<Q, S, MT_COLL_LBGK><<<grid_for(lv.nfused, B), B, 0, s>>>(
                        lv.fused_list, lv.nfused, n, tb, lv.nbr, A::fcol(lv), A::f(lv), (S *)lv.fcol_alt,
                        c.d.tau[l], A::rho(lv), A::u(lv), mac, c.shift[l]);
                } else {
                    if constexpr (Q == 27)
                        k_pull_collide<Q, S, MT_COLL_CUMULANT><<<grid_for(lv.nfused, 64), 64, 0, s>>>(
                            lv.fused_list, lv.nfused, n, tb, lv.nbr, A::fcol(lv), A::f(lv), (S *)lv.fcol_alt,
                            c.d.tau[l], A::rho(lv), A::u(lv), mac, c.shift[l]);
                }
                MT_LAUNCHED(ctx);
            }
            if (lv.nlist[2]) {
                k_pull_copy<Q, S><<<grid_for(lv.nlist[2], B), B, 0, s>>>(lv.list[2], lv.nlist[2], n, tb, lv.nbr,
                                                                          A::fcol(lv), A::f(lv), (S *)lv.fcol_alt);
                MT_LAUNCHED(ctx);
            }
            if (lv.nband) {
                k_stream<Q, S><<<grid_for(lv.nband, B), B, 0, s>>>(lv.band, lv.nband, n, tb, lv.nbr, A::fcol(lv),
                                                                    A::f(lv));
                MT_LAUNCHED(ctx);
            }
        }
        if (is != s) {
            MT_CUDA(ctx, cudaEventRecord(c.ev_join, is));
            MT_CUDA(ctx, cudaStreamWaitEvent(s, c.ev_join, 0));
        }
        return MT_OK;
    }
    }
    return set_err(ctx, MT_ERR_ARG, "unknown phase");
}

template <class S>
int AmrOps<S>::phase(Ctx &ctx, Case &c, int phase, int level)
{
    return c.d.q == 19 ? amr_phase_q<S, 19>(ctx, c, phase, level) : amr_phase_q<S, 27>(ctx, c, phase, level);
}

template <class S>
int AmrOps<S>::upload_tables(Ctx &ctx)
{
    return upload_bdry_tables(ctx);
}

template <class S>
int AmrOps<S>::alloc(Ctx &ctx, Case &c, int l)
{
    using C = typename Store<S>::C;
    Level &lv = c.lv[l];
    const int64_t n = lv.n, Q = c.d.q;
    if (l == 0) {
        int rc = upload_bdry_tables(ctx);
        if (rc) return rc;
    }
    lv.brick_variant = brick_default_variant<S>();
    MT_CUDA(ctx, cudaMallocAsync(&lv.f, sizeof(S) * n * Q, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&lv.fcol, sizeof(S) * n * Q, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&lv.rho, sizeof(C) * n, ctx.stream));
    MT_CUDA(ctx, cudaMallocAsync(&lv.u, sizeof(C) * 3 * n, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.f, 0, sizeof(S) * n * Q, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.fcol, 0, sizeof(S) * n * Q, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.rho, 0, sizeof(C) * n, ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(lv.u, 0, sizeof(C) * 3 * n, ctx.stream));
    return MT_OK;
}

template <class S>
int AmrOps<S>::init_eq(Ctx &ctx, Case &c, double rho0, const double *u0)
{
    using A = AmrTyped<S>;
    for (int l = 0; l <= c.d.max_level; ++l) {
        Level &lv = c.lv[l];
        if (!lv.n) continue;
        if (c.d.q == 19)
            k_init_eq<19, S><<<grid_for(lv.n, 256), 256, 0, ctx.stream>>>(lv.n, lv.tag, rho0, u0[0], u0[1], u0[2],
                                                                           A::f(lv), A::fcol(lv), A::rho(lv), A::u(lv), c.shift[l]);
        else
            k_init_eq<27, S><<<grid_for(lv.n, 256), 256, 0, ctx.stream>>>(lv.n, lv.tag, rho0, u0[0], u0[1], u0[2],
                                                                           A::f(lv), A::fcol(lv), A::rho(lv), A::u(lv), c.shift[l]);
        MT_LAUNCHED(ctx);
    }
    return MT_OK;
}

template <class S>
int AmrOps<S>::get(Ctx &ctx, Case &c, int l, int which, double *d_out)
{
    Level &lv = c.lv[l];
    const S *src = (const S *)(which == 0 ? lv.f : lv.fcol);
    if (!lv.n) return MT_OK;
    if (c.d.q == 19)
        k_to_f64<19, S><<<grid_for(lv.n, 256), 256, 0, ctx.stream>>>(src, d_out, lv.n, c.shift[l]);
    else
        k_to_f64<27, S><<<grid_for(lv.n, 256), 256, 0, ctx.stream>>>(src, d_out, lv.n, c.shift[l]);
    MT_LAUNCHED(ctx);
    return MT_OK;
}

template <class S>
int AmrOps<S>::set(Ctx &ctx, Case &c, int l, int which, const double *d_in)
{
    Level &lv = c.lv[l];
    S *dst = (S *)(which == 0 ? lv.f : lv.fcol);
    if (!lv.n) return MT_OK;
    if (c.d.q == 19)
        k_from_f64<19, S><<<grid_for(lv.n, 256), 256, 0, ctx.stream>>>(d_in, dst, lv.n, c.shift[l]);
    else
        k_from_f64<27, S><<<grid_for(lv.n, 256), 256, 0, ctx.stream>>>(d_in, dst, lv.n, c.shift[l]);
    MT_LAUNCHED(ctx);
    return MT_OK;
}

template <class S>
int AmrOps<S>::macros_out(Ctx &ctx, Case &c, int l, double *d_rho, double *d_u)
{
    using C = typename Store<S>::C;
    Level &lv = c.lv[l];
    if (!lv.n) return MT_OK;
    k_macro_to_f64<C><<<grid_for(lv.n, 256), 256, 0, ctx.stream>>>((const C *)lv.rho, d_rho, lv.n);
    MT_LAUNCHED(ctx);
    k_macro_to_f64<C><<<grid_for(3 * lv.n, 256), 256, 0, ctx.stream>>>((const C *)lv.u, d_u, 3 * lv.n);
    MT_LAUNCHED(ctx);
    return MT_OK;
}

template <class S>
int AmrOps<S>::batch_pass(Ctx &ctx, int q, int coll, const BrickBatch *d_desc, int64_t total, const Shift &sh)
{
    const unsigned g = grid_for(total, 4);
    if (!g) return MT_OK;
    constexpr int V = brick_default_variant<S>();
    if (q == 19)
        k_brick_step_batch<19, S, MT_COLL_LBGK, V><<<g, 128, 0, ctx.stream>>>(d_desc, sh);
    else if (coll == MT_COLL_LBGK)
        k_brick_step_batch<27, S, MT_COLL_LBGK, V><<<g, 128, 0, ctx.stream>>>(d_desc, sh);
    else
        k_brick_step_batch<27, S, MT_COLL_CUMULANT, V><<<g, 128, 0, ctx.stream>>>(d_desc, sh);
    MT_LAUNCHED(ctx);
    return MT_OK;
}

// ---- the brick pass autotuner (mt_case_tune_bricks) ----------------------
// Each brick level's fused pass is timed in each of its forms (0 one cell per
// lane step at 8 resident blocks per SM; 1 two cells with packed FP32 pairs;
// 2 one cell at 6 blocks with more registers; 3 the lane's two cells in one
// unrolled sequence at 6 blocks; FP64 has forms 0 and 3) on the case's own
// bricks: one warm-up and three timed launches per form, CUDA
// events on the case's stream.  The passes read the current post-collision
// buffer and write the next collision into a scratch buffer; the f they
// store is what the last real pass stored, and no macros are written, so the
// state is untouched.  The faster form is kept for the level.
template <class S>
int AmrOps<S>::tune_bricks(Ctx &ctx, Case &c, int32_t *variant, float *ms)
{
    int64_t nmax = 0;
    for (int l = 0; l <= c.d.max_level; ++l)
        if (c.lv[l].bricks) nmax = std::max(nmax, c.lv[l].n);
    for (int l = 0; l <= c.d.max_level; ++l) {
        if (variant) variant[l] = -1;
        if (ms)
            for (int v = 0; v < MT_BRICK_FORMS; ++v) ms[MT_BRICK_FORMS * l + v] = -1.f;
    }
    if (!nmax) return MT_OK;
    S *scratch = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&scratch, sizeof(S) * (size_t)c.d.q * (size_t)nmax, ctx.stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = MT_OK;
    for (int l = 0; l <= c.d.max_level && !rc; ++l) {
        Level &lv = c.lv[l];
        if (!lv.bricks || !lv.nbrick) continue;
        float best = 0.f;
        int pick = lv.brick_variant;
        for (int v = 0; v < MT_BRICK_FORMS && !rc; ++v) {
            if (!Store<S>::shifted && v != 0 && v != 3) continue;  // FP64: forms 0 and 3
            auto launch = [&]() {
                if (c.d.q == 19)
                    brick_launch<19, S>(c, l, v, ctx.stream, scratch, 0, 0, nullptr);
                else
                    brick_launch<27, S>(c, l, v, ctx.stream, scratch, 0, 0, nullptr);
            };
            launch();
            cudaEventRecord(e0, ctx.stream);
            for (int r = 0; r < 3; ++r) launch();
            cudaEventRecord(e1, ctx.stream);
            cudaError_t e = cudaEventSynchronize(e1);
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e != cudaSuccess) {
                rc = set_err(ctx, MT_ERR_CUDA, std::string("brick tuner: ") + cudaGetErrorString(e));
                break;
            }
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            t /= 3.f;
            ctx.launches += 4;
            if (ms) ms[MT_BRICK_FORMS * l + v] = t;
            if (v == 0 || t < best) {  // form 0 is always timed first
                best = t;
                pick = v;
            }
        }
        lv.brick_variant = pick;
        if (variant) variant[l] = pick;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(scratch, ctx.stream);
    return rc;
}

// ---- FP64 reductions of a multi-level case (mt_case_reduce_levels) -------
// Per-block partial sums over a level's stepped cells (the collide list,
// lat_f then overlap_F2C: the cells LBM_Manager::calculateMacros visits,
// LBM_Manager.cpp:1003-1050) of mass sum_q f_q, momentum sum_q f_q e_q and
// kinetic energy |j|^2 / (2 rho), every value widened to FP64 before the
// storage shift (FP64) is added back.  partial: [5][gridDim.x].
template <int Q, class S>
__global__ void k_level_reduce(const S *f, int64_t n, const int32_t *list, int64_t m, const Shift sh,
                               double *partial)
{
    __shared__ double red[5][256];
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double a[5] = {0, 0, 0, 0, 0};
    if (j < m) {
        const int64_t i = list[j];
        double r = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            double v = (double)Store<S>::ld(f, (int64_t)k * n + i);
            if (Store<S>::shifted) v += sh.d[k];
            r += v;
            jx += v * ex(k);
            jy += v * ey(k);
            jz += v * ez(k);
        }
        a[0] = r;
        a[1] = jx;
        a[2] = jy;
        a[3] = jz;
        a[4] = 0.5 * (jx * jx + jy * jy + jz * jz) / r;
    }
    for (int c = 0; c < 5; ++c) red[c][threadIdx.x] = a[c];
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            for (int c = 0; c < 5; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 5; ++c) partial[(int64_t)c * gridDim.x + blockIdx.x] = red[c][0];
}

// where each level's partials start in the scratch and how many blocks it has
struct LevelPartials {
    int64_t off[kMaxLevels];
    int64_t nb[kMaxLevels];
    int nlev;
};

// one block: level rows in a fixed order (strided sums, then a tree), then
// the global row sum_l 8^-l row_l (a level-l cell is 8^-l coarse cells).
// out: [(nlev + 1) * 5]
static __global__ void k_level_totals(const double *partial, const LevelPartials P, double *out)
{
    __shared__ double red[256];
    for (int l = 0; l < P.nlev; ++l)
        for (int c = 0; c < 5; ++c) {
            const double *p = partial + P.off[l] + (int64_t)c * P.nb[l];
            double a = 0;
            for (int64_t j = threadIdx.x; j < P.nb[l]; j += blockDim.x) a += p[j];
            red[threadIdx.x] = a;
            __syncthreads();
            for (int st = blockDim.x / 2; st > 0; st >>= 1) {
                if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
                __syncthreads();
            }
            if (threadIdx.x == 0) out[l * 5 + c] = red[0];
            __syncthreads();
        }
    if (threadIdx.x < 5) {
        double g = 0, wl = 1.0;
        for (int l = 0; l < P.nlev; ++l) {
            g += wl * out[l * 5 + threadIdx.x];
            wl *= 0.125;
        }
        out[P.nlev * 5 + threadIdx.x] = g;
    }
}

template <class S>
int AmrOps<S>::reduce(Ctx &ctx, Case &c, double *d_out)
{
    LevelPartials P{};
    P.nlev = c.d.max_level + 1;
    int64_t total = 0;
    for (int l = 0; l < P.nlev; ++l) {
        P.off[l] = total;
        P.nb[l] = (c.lv[l].ncollide + 255) / 256;
        total += 5 * P.nb[l];
    }
    double *partial = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&partial, sizeof(double) * std::max<int64_t>(total, 1), ctx.stream));
    cudaError_t err = cudaSuccess;
    auto launched = [&]() {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) err = e;
        else ctx.launches++;
        return e == cudaSuccess;
    };
    bool ok = true;
    for (int l = 0; l < P.nlev && ok; ++l) {
        Level &lv = c.lv[l];
        if (!P.nb[l]) continue;
        if (c.d.q == 19)
            k_level_reduce<19, S><<<(unsigned)P.nb[l], 256, 0, ctx.stream>>>(
                (const S *)lv.f, lv.n, lv.collide_list, lv.ncollide, c.shift[l], partial + P.off[l]);
        else
            k_level_reduce<27, S><<<(unsigned)P.nb[l], 256, 0, ctx.stream>>>(
                (const S *)lv.f, lv.n, lv.collide_list, lv.ncollide, c.shift[l], partial + P.off[l]);
        ok = launched();
    }
    if (ok) {
        k_level_totals<<<1, 256, 0, ctx.stream>>>(partial, P, d_out);
        ok = launched();
    }
    cudaFreeAsync(partial, ctx.stream);
    if (!ok) return set_err(ctx, MT_ERR_CUDA, std::string("reduction launch: ") + cudaGetErrorString(err));
    return MT_OK;
}

// ---- LBM_Manager::infoPrint's diagnostics (mt_case_info) ----------------
// Per block over a level's collide list (lat_f then overlap_F2C, the cells
// infoPrint visits, LBM_Manager.cpp:914-955): the largest |u| and the number
// of cells with |u| > 1 over both sets, and over the lat_f cells (the first
// nlatf entries) sum |u - u_prev|^2 and sum |u|^2, u_prev the velocity the
// previous call saw (prev [3][nlatf], FP64, rewritten here).  A NaN velocity
// never wins the maximum, as in the reference's comparisons.
// partial: [4][gridDim.x]
template <class C>
__global__ void k_level_info(const int32_t *__restrict__ list, int64_t m, int64_t nlatf, const C *__restrict__ u,
                             int64_t n, double *__restrict__ prev, int have_prev, double *__restrict__ partial)
{
    __shared__ double red[4][256];
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double a[4] = {0, 0, 0, 0};
    if (j < m) {
        const int64_t i = list[j];
        const double ux = (double)u[i], uy = (double)u[n + i], uz = (double)u[2 * n + i];
        const double v2 = ux * ux + uy * uy + uz * uz;
        const double vmag = sqrt(v2);
        a[0] = vmag > 0.0 ? vmag : 0.0;
        a[1] = vmag > 1.0 ? 1.0 : 0.0;
        if (j < nlatf) {
            if (have_prev) {
                const double dx = ux - prev[j], dy = uy - prev[nlatf + j], dz = uz - prev[2 * nlatf + j];
                a[2] = dx * dx + dy * dy + dz * dz;
            }
            a[3] = v2;
            prev[j] = ux;
            prev[nlatf + j] = uy;
            prev[2 * nlatf + j] = uz;
        }
    }
    for (int c = 0; c < 4; ++c) red[c][threadIdx.x] = a[c];
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) {
            red[0][threadIdx.x] = fmax(red[0][threadIdx.x], red[0][threadIdx.x + st]);
            for (int c = 1; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + st];
        }
        __syncthreads();
    }
    if (threadIdx.x < 4) partial[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = red[threadIdx.x][0];
}

// one block: each level's row (column 0 the maximum, the others sums) in a
// fixed order.  out: [nlev * 4]
static __global__ void k_info_totals(const double *partial, const LevelPartials P, double *out)
{
    __shared__ double red[256];
    for (int l = 0; l < P.nlev; ++l)
        for (int c = 0; c < 4; ++c) {
            const double *p = partial + P.off[l] + (int64_t)c * P.nb[l];
            double a = 0;
            for (int64_t j = threadIdx.x; j < P.nb[l]; j += blockDim.x) a = c == 0 ? fmax(a, p[j]) : a + p[j];
            red[threadIdx.x] = a;
            __syncthreads();
            for (int st = blockDim.x / 2; st > 0; st >>= 1) {
                if (threadIdx.x < st)
                    red[threadIdx.x] = c == 0 ? fmax(red[threadIdx.x], red[threadIdx.x + st])
                                              : red[threadIdx.x] + red[threadIdx.x + st];
                __syncthreads();
            }
            if (threadIdx.x == 0) out[l * 4 + c] = red[0];
            __syncthreads();
        }
}

template <class S>
int AmrOps<S>::info(Ctx &ctx, Case &c, double *d_out)
{
    using C = typename Store<S>::C;
    LevelPartials P{};
    P.nlev = c.d.max_level + 1;
    int64_t total = 0;
    for (int l = 0; l < P.nlev; ++l) {
        P.off[l] = total;
        P.nb[l] = (c.lv[l].ncollide + 255) / 256;
        total += 4 * P.nb[l];
        Level &lv = c.lv[l];
        if (!lv.info_prev && lv.nlist[0])
            MT_CUDA(ctx, cudaMallocAsync(&lv.info_prev, sizeof(double) * 3 * (size_t)lv.nlist[0], ctx.stream));
    }
    double *partial = nullptr;
    MT_CUDA(ctx, cudaMallocAsync(&partial, sizeof(double) * std::max<int64_t>(total, 1), ctx.stream));
    MT_CUDA(ctx, cudaMemsetAsync(d_out, 0, sizeof(double) * 4 * (size_t)P.nlev, ctx.stream));
    cudaError_t err = cudaSuccess;
    bool ok = true;
    for (int l = 0; l < P.nlev && ok; ++l) {
        Level &lv = c.lv[l];
        if (!P.nb[l]) continue;
        k_level_info<C><<<(unsigned)P.nb[l], 256, 0, ctx.stream>>>(lv.collide_list, lv.ncollide, lv.nlist[0],
                                                                 AmrTyped<S>::u(lv), lv.n, lv.info_prev,
                                                                 lv.info_have ? 1 : 0, partial + P.off[l]);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            err = e;
            ok = false;
        } else {
            ctx.launches++;
            lv.info_have = true;
        }
    }
    if (ok) {
        k_info_totals<<<1, 256, 0, ctx.stream>>>(partial, P, d_out);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            err = e;
            ok = false;
        } else {
            ctx.launches++;
        }
    }
    cudaFreeAsync(partial, ctx.stream);
    if (!ok) return set_err(ctx, MT_ERR_CUDA, std::string("info launch: ") + cudaGetErrorString(err));
    return MT_OK;
}


template <class S>
int AmrOps<S>::guard(Ctx &ctx, Case &c, bool current_only)
{
    for (int l = 0; l <= c.d.max_level; ++l) {
        Level &lv = c.lv[l];
        if (!lv.n) continue;
        const int64_t total = lv.n * c.d.q;
        k_guard<S><<<(unsigned)std::min<int64_t>(grid_for(total, 256), 148 * 16), 256, 0, ctx.stream>>>(
            (const S *)(current_only ? lv.fcol : lv.f), (const S *)lv.fcol, total, c.dev_err);
        MT_LAUNCHED(ctx);
    }
    return MT_OK;
}

// ---- remap of a state onto another lattice (mt_case_remap) ---------------
// one population set of Q values rescaled about its own equilibrium:
// feq(rho, u) + s (in - feq(rho, u)), rho and u from the values themselves
template <int Q> __device__ void remap_rescale(double *v, double s)
{
    double r = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
    for (int k = 0; k < Q; ++k) {
        r += v[k];
        jx += v[k] * ex(k);
        jy += v[k] * ey(k);
        jz += v[k] * ez(k);
    }
    const double rs = (r > -1e-6 && r < 1e-6) ? ((r < 0.0) ? -1e-6 : 1e-6) : r;
    const double ux = jx / rs, uy = jy / rs, uz = jz / rs;
    const double uu = ux * ux + uy * uy + uz * uz;
    for (int k = 0; k < Q; ++k) {
        const double eu = ex(k) * ux + ey(k) * uy + ez(k) * uz;
        const double feq = r * w<Q>(k) * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uu);
        v[k] = feq + s * (v[k] - feq);
    }
}

__host__ __device__ __forceinline__ uint64_t cell_key_at(int L, int l, int64_t x, int64_t y, int64_t z)
{
    const int sh = L - l;
    return dilate3((uint64_t)x << sh) | (dilate3((uint64_t)y << sh) << 1) | (dilate3((uint64_t)z << sh) << 2);
}

template <class S> struct RemapLevels {
    struct Src {
        const uint64_t *key = nullptr;
        const uint32_t *tag = nullptr;
        int64_t n = 0;
        const S *f = nullptr, *fcol = nullptr;
        float shift[27] = {};  // the level's storage shift (reduced storages)
    } lv[kMaxLevels];
    // explosion factors from coarser source level m, coalescence factors
    // from finer source level m (products over the levels crossed)
    double up_f[kMaxLevels], up_c[kMaxLevels], down_f[kMaxLevels], down_c[kMaxLevels];
};

// Each cell of a destination level takes f and fcol from the source: the same
// key on the same level as they are (the stored values, bit for bit); else
// the nearest coarser source level holding its ancestor, rescaled as an
// explosion; else the mean of its descendants on the nearest finer source
// level holding any, rescaled as a coalescence; else the equilibrium
// (rho0, u0).  Solid cells hold zeros (the build's convention); a fluid cell
// that is solid in the source takes the equilibrium at rest.  kind[i]: 0..3.
template <int Q, class S>
__global__ void k_remap(const uint64_t *dkey, const uint32_t *dtag, int64_t nd, int L, int l, RemapLevels<S> src,
                        double rho0, double ux0, double uy0, double uz0, S *fo, S *co, uint8_t *kind, const Shift dsh,
                        int same_shift)
{
    using T = Store<S>;
    using C = typename T::C;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nd) return;
    const uint64_t k = dkey[i];
    double a[Q], b[Q];
    auto put = [&](const double *pf, const double *pc, int kd) {
        for (int q = 0; q < Q; ++q) {
            T::st(fo, q * nd + i, stored_sh<S>(dsh, (C)pf[q], q));
            T::st(co, q * nd + i, stored_sh<S>(dsh, (C)pc[q], q));
        }
        kind[i] = (uint8_t)kd;
    };
    if (dtag[i] & TAG_SF) {
        for (int q = 0; q < Q; ++q) a[q] = 0.0;
        put(a, a, 0);
        return;
    }
    const auto &same = src.lv[l];
    int64_t j = same.n ? find_key(same.key, same.n, k) : -1;
    bool uncovered = false;
    if (j >= 0 && (same.tag[j] & TAG_SF)) {
        uncovered = true;
        j = -1;
    }
    if (j >= 0) {
        if (same_shift) {
            for (int q = 0; q < Q; ++q) {
                fo[q * nd + i] = same.f[q * same.n + j];
                co[q * nd + i] = same.fcol[q * same.n + j];
            }
        } else {
            for (int q = 0; q < Q; ++q) {
                T::st(fo, q * nd + i, stored_sh<S>(dsh, full_v<S>(same.shift, T::ld(same.f, q * same.n + j), q), q));
                T::st(co, q * nd + i, stored_sh<S>(dsh, full_v<S>(same.shift, T::ld(same.fcol, q * same.n + j), q), q));
            }
        }
        kind[i] = 0;
        return;
    }
    const int sh = L - l;
    const int64_t x = (int64_t)(compact3(k) >> sh), y = (int64_t)(compact3(k >> 1) >> sh),
                  z = (int64_t)(compact3(k >> 2) >> sh);
    for (int m = l - 1; m >= 0 && !uncovered; --m) {
        const auto &cs = src.lv[m];
        if (!cs.n) continue;
        const int up = l - m;
        const int64_t jm = find_key(cs.key, cs.n, cell_key_at(L, m, x >> up, y >> up, z >> up));
        if (jm < 0) continue;
        for (int q = 0; q < Q; ++q) {
            a[q] = (double)full_v<S>(cs.shift, T::ld(cs.f, q * cs.n + jm), q);
            b[q] = (double)full_v<S>(cs.shift, T::ld(cs.fcol, q * cs.n + jm), q);
        }
        remap_rescale<Q>(a, src.up_f[m]);
        remap_rescale<Q>(b, src.up_c[m]);
        put(a, b, 1);
        return;
    }
    for (int d = 1; l + d <= L && !uncovered; ++d) {
        const auto &fine = src.lv[l + d];
        if (!fine.n) continue;
        const int side = 1 << d;
        int nch = 0;
        for (int q = 0; q < Q; ++q) a[q] = b[q] = 0.0;
        for (int c = 0; c < side * side * side; ++c) {
            const int64_t cx = (x << d) + c % side, cy = (y << d) + (c / side) % side, cz = (z << d) + c / (side * side);
            const int64_t jc = find_key(fine.key, fine.n, cell_key_at(L, l + d, cx, cy, cz));
            if (jc < 0 || (fine.tag[jc] & TAG_SF)) continue;
            for (int q = 0; q < Q; ++q) {
                a[q] += (double)full_v<S>(fine.shift, T::ld(fine.f, q * fine.n + jc), q);
                b[q] += (double)full_v<S>(fine.shift, T::ld(fine.fcol, q * fine.n + jc), q);
            }
            ++nch;
        }
        if (!nch) continue;
        for (int q = 0; q < Q; ++q) {
            a[q] /= nch;
            b[q] /= nch;
        }
        remap_rescale<Q>(a, src.down_f[l + d]);
        remap_rescale<Q>(b, src.down_c[l + d]);
        put(a, b, 2);
        return;
    }
    if (uncovered) ux0 = uy0 = uz0 = 0.0;
    const double uu = ux0 * ux0 + uy0 * uy0 + uz0 * uz0;
    for (int q = 0; q < Q; ++q) {
        const double eu = ex(q) * ux0 + ey(q) * uy0 + ez(q) * uz0;
        a[q] = rho0 * w<Q>(q) * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uu);
    }
    put(a, a, 3);
}

template <class S>
int AmrOps<S>::remap(Ctx &ctx, Case &dst, Case &src, int64_t *counts)
{
    const int L = dst.d.max_level, Q = dst.d.q;
    RemapLevels<S> rl;
    for (int m = 0; m <= L && m <= src.d.max_level; ++m) {
        if (!src.lv[m].n) continue;
        rl.lv[m].key = src.lv[m].key;
        rl.lv[m].tag = src.lv[m].tag;
        rl.lv[m].n = src.lv[m].n;
        rl.lv[m].f = (const S *)src.lv[m].f;
        rl.lv[m].fcol = (const S *)src.lv[m].fcol;
        for (int k = 0; k < 27; ++k) rl.lv[m].shift[k] = src.shift[m].v[k];
    }
    // the interface factors of dst: the reference's (the same on f and
    // fcol), or the stress-continuous ones (tau on f, tau - 1 on fcol)
    const bool st = dst.scaling == MT_SCALE_STANDARD;
    auto c2f = [&](int fine, bool col) {
        const double tf = dst.d.tau[fine], tc = dst.d.tau[fine - 1];
        if (!st) return (2.0 * tf) / tc;
        return col ? (tf - 1.0) / (2.0 * (tc - 1.0)) : tf / (2.0 * tc);
    };
    uint8_t *kind = nullptr;
    int64_t maxn = 0;
    for (int l = 0; l <= L; ++l) maxn = std::max(maxn, dst.lv[l].n);
    MT_CUDA(ctx, cudaMallocAsync(&kind, std::max<int64_t>(maxn, 1), ctx.stream));
    int rc = MT_OK;
    for (int l = 0; l <= L && !rc; ++l) {
        Level &lv = dst.lv[l];
        if (counts)
            for (int k = 0; k < 4; ++k) counts[4 * l + k] = 0;
        if (!lv.n) continue;
        for (int m = 0; m < kMaxLevels; ++m) rl.up_f[m] = rl.up_c[m] = rl.down_f[m] = rl.down_c[m] = 1.0;
        for (int m = l - 1; m >= 0; --m)
            for (int j = m + 1; j <= l; ++j) {
                rl.up_f[m] *= c2f(j, false);
                rl.up_c[m] *= c2f(j, true);
            }
        for (int m = l + 1; m <= L; ++m)
            for (int j = l + 1; j <= m; ++j) {
                rl.down_f[m] /= c2f(j, false);
                rl.down_c[m] /= c2f(j, true);
            }
        const double r0 = dst.d.rho0, u0 = dst.d.u_bc[0], u1 = dst.d.u_bc[1], u2 = dst.d.u_bc[2];
        // equal storage shifts on level l: cells present on both lattices copy their stored values
        int same_shift = l <= src.d.max_level;
        for (int k = 0; k < 27; ++k) same_shift &= dst.shift[l].d[k] == src.shift[l].d[k];
        if (Q == 19)
            k_remap<19, S><<<grid_for(lv.n, 128), 128, 0, ctx.stream>>>(lv.key, lv.tag, lv.n, L, l, rl, r0, u0, u1, u2,
                                                                       (S *)lv.f, (S *)lv.fcol, kind, dst.shift[l],
                                                                       same_shift);
        else
            k_remap<27, S><<<grid_for(lv.n, 128), 128, 0, ctx.stream>>>(lv.key, lv.tag, lv.n, L, l, rl, r0, u0, u1, u2,
                                                                       (S *)lv.f, (S *)lv.fcol, kind, dst.shift[l],
                                                                       same_shift);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            rc = set_err(ctx, MT_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
            break;
        }
        ctx.launches++;
        if (counts) {
            std::vector<uint8_t> hk((size_t)lv.n);
            e = cudaMemcpyAsync(hk.data(), kind, lv.n, cudaMemcpyDeviceToHost, ctx.stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
            if (e != cudaSuccess) {
                rc = set_err(ctx, MT_ERR_CUDA, std::string("remap counts: ") + cudaGetErrorString(e));
                break;
            }
            for (uint8_t v : hk) counts[4 * l + (v & 3)] += 1;
        }
    }
    cudaFreeAsync(kind, ctx.stream);
    return rc;
}

}  // namespace mt
