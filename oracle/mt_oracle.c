/*
 * mt_oracle.c -- CPU restatement (FP64) of the multi-level lattice-Boltzmann
 * time step of MortonTrieCode-CAD2025/mortonTrie_AMR.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * it.  The product library never links or calls it.
 *
 * Parity is pinned against the reference itself: oracle/refharness drives
 * the reference's own LBM translation units on the same index sets and the
 * golden files under tests/golden/ hold its outputs.  The restated boundary
 * conditions that have no runnable reference code (periodic wrap, ZouHe
 * velocity inlet, zero-gradient outflow) are parity-unpinned.
 *
 * Every floating-point expression keeps the reference's operation order so
 * that the FP64 results match it bit-for-bit when compiled without FMA
 * contraction (-ffp-contract=off; g++ -O3 on x86-64 emits no FMA either).
 *
 * Data model: per level, the union of all index sets sorted by Morton key;
 * populations are structure-of-arrays f[q*n + i].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OC_MAXL 8
#define OC_NSETS 6

enum { S_LATF = 0, S_F2C = 1, S_C2F = 2, S_GC2F = 3, S_GF2C = 4, S_SF = 5, S_BAND = 6, S_BC0 = 16 };
enum { T_LATF = 1, T_F2C = 2, T_C2F = 4, T_GC2F = 8, T_GF2C = 16, T_BC = 32, T_SF = 64, T_IB = 128, T_BAND = 256 };
enum { COLL_LBGK = 0, COLL_CUMULANT = 1 };
enum { IB_DW = 0, IB_FH = 1, IB_DF = 2 };
/* domain boundary treatment on the x faces (the y/z faces follow the same
 * rule when they are not periodic) */
enum { BC_NEQ = 0, BC_ZOUHE_OUTFLOW = 1, BC_ZOUHE_HH = 2 };

/* Lattice tables in the reference ordering (header/Constants.h:492-538). */
static const int EX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0,
                           1, -1, 1, -1, -1, 1, -1, 1};
static const int EY[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1,
                           1, -1, -1, 1, -1, 1, 1, -1};
static const int EZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1,
                           1, -1, 1, -1, 1, -1, 1, -1};
static const int INV[27] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17,
                            20, 19, 22, 21, 24, 23, 26, 25};

/* Reserved (inward/tangential) directions per boundary set, D3Q19 and D3Q27
 * (D3Q19_BC_Manager.hpp:60-122). */
static const int BDRY19[26][14] = {
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
static const int BDRY27[26][18] = {
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

/* Face groups in the order the reference applies them after streaming
 * (LBM_Simulator.cpp:90-95: West, East, South, North, Bot, Top) with the
 * boundary sets each group owns (NonEquilibrumExtrapolation.hpp:24-110). */
static const int FACE_SETS[6][9] = {
    {0, 7, 8, 15, 17, 19, 20, 23, 24}, {1, 6, 9, 14, 16, 18, 21, 22, 25},
    {2, 11, 13, -1, -1, -1, -1, -1, -1}, {3, 10, 12, -1, -1, -1, -1, -1, -1},
    {4, -1, -1, -1, -1, -1, -1, -1, -1}, {5, -1, -1, -1, -1, -1, -1, -1, -1}};

typedef struct {
    uint64_t *keys;
    int64_t n, cap;
} keyvec;

typedef struct {
    int64_t n;
    uint64_t *key;
    uint32_t *tag;
    int8_t *bcidx;
    int32_t *disrow;
    double *f, *fcol, *rho, *u;
    int64_t nlist[OC_NSETS];
    int64_t *list[OC_NSETS];
    int64_t nbc[26];
    int64_t *bclist[26];
    keyvec raw[OC_NSETS];
    keyvec rawbc[26];
    keyvec rawband;
    int64_t nband;
    int64_t *band;
    double *prev; /* MT_ITIME_EXTRAP: explosion sources' parent values at the previous parent step */
} oc_level;

typedef struct {
    int q, L, collision, ib_method, bc_mode, stream_conv;
    int itime; /* 0 explosion in the first substep, 1 hold, 2 extrapolated second substep */
    int prev_stale; /* the saved sources no longer belong to the state */
    int periodic[3];
    int64_t extent0[3];
    double tau[OC_MAXL];
    double rho0, u_bc[3];
    double face_u[6][3]; /* bc_velocity of each face strategy */
    oc_level lv[OC_MAXL];
    int64_t ndis;
    uint64_t *dis_key;
    double *dis;
    double fx, fy, fz;
    int64_t nforce;
    int built;
    /* direct-forcing markers (finest-level cell units) */
    int64_t nm, period, tstep;
    double *mref, *mdv, *path, center[3];
    int64_t *acc; /* [3][n_L] Eulerian force in fixed point 2^-32 */
} oc_case;

/* ------------------------------------------------------------------ */
/* Morton neighbour arithmetic (Morton_Assist.h:229-289,              */
/* Morton_Assist.cpp:20-106): masked increment/decrement of one axis's  */
/* bits at or above the level bit; x, then y, then z.                   */
/* ------------------------------------------------------------------ */
static uint64_t axis_mask(int L, int level, int axis)
{
    /* bits of `axis` at positions >= 3(L-level), up to the last whole
     * 3-bit group that fits below bit 63 */
    uint64_t m = 0;
    int nbg = (64 - 3 * L) / 3;
    for (int k = L - level; k < L + nbg; ++k) {
        int p = 3 * k + axis;
        if (p < 64) m |= (uint64_t)1 << p;
    }
    return m;
}

static uint64_t axis_fill(int L, int level, int axis)
{
    /* complement of the axis mask restricted to bits >= 3(L-level) */
    uint64_t m = ~axis_mask(L, level, axis);
    int lowbits = 3 * (L - level);
    if (lowbits > 0) m &= ~(((uint64_t)1 << lowbits) - 1);
    return m;
}

static uint64_t compact3(uint64_t v)
{
    v &= 0x1249249249249249ULL;
    v = (v ^ (v >> 2)) & 0x10C30C30C30C30C3ULL;
    v = (v ^ (v >> 4)) & 0x100F00F00F00F00FULL;
    v = (v ^ (v >> 8)) & 0x1F0000FF0000FFULL;
    v = (v ^ (v >> 16)) & 0x1F00000000FFFFULL;
    v = (v ^ (v >> 32)) & 0x1FFFFFULL;
    return v;
}

static uint64_t dilate3(uint64_t v)
{
    v &= 0x1FFFFFULL;
    v = (v | (v << 32)) & 0x1F00000000FFFFULL;
    v = (v | (v << 16)) & 0x1F0000FF0000FFULL;
    v = (v | (v << 8)) & 0x100F00F00F00F00FULL;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ULL;
    v = (v | (v << 2)) & 0x1249249249249249ULL;
    return v;
}

/* one axis step, +1 or -1, on a key of level `level` */
static uint64_t axis_step(const oc_case *c, uint64_t key, int level, int axis, int dir)
{
    int L = c->L;
    uint64_t m1 = axis_mask(L, level, axis);
    uint64_t others = 0;
    for (int a = 0; a < 3; ++a)
        if (a != axis) others |= key & axis_mask(L, level, a);
    if (c->periodic[axis]) {
        int64_t ext = c->extent0[axis] << level;
        int sh = L - level;
        int64_t coord = (int64_t)(compact3(key >> axis) >> sh);
        coord += dir;
        if (coord < 0) coord += ext;
        if (coord >= ext) coord -= ext;
        return ((dilate3((uint64_t)coord << sh) << axis) & m1) | others;
    }
    uint64_t one = (uint64_t)1 << (3 * (L - level) + axis);
    uint64_t t;
    if (dir > 0)
        t = (key | axis_fill(L, level, axis)) + one;
    else
        t = (key & m1) - one;
    return (t & m1) | others;
}

static uint64_t find_neighbor(const oc_case *c, uint64_t key, int level, int dx, int dy, int dz)
{
    uint64_t r = key;
    if (dx) r = axis_step(c, r, level, 0, dx);
    if (dy) r = axis_step(c, r, level, 1, dy);
    if (dz) r = axis_step(c, r, level, 2, dz);
    return r;
}

static int64_t find_sorted(const uint64_t *k, int64_t n, uint64_t key)
{
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = lo + ((hi - lo) >> 1);
        if (k[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < n && k[lo] == key) ? lo : -1;
}

static int64_t find_idx(const oc_level *lv, uint64_t key)
{
    int64_t lo = 0, hi = lv->n;
    while (lo < hi) {
        int64_t mid = lo + ((hi - lo) >> 1);
        if (lv->key[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < lv->n && lv->key[lo] == key) ? lo : -1;
}

/* ------------------------------------------------------------------ */
/* Equilibria and macros (LBM_Manager.cpp:137-263, 983-1001)           */
/* ------------------------------------------------------------------ */
static double wq(int q, int i)
{
    if (q == 19) {
        if (i == 0) return 1. / 3.;
        if (i <= 6) return 1. / 18.;
        return 1. / 36.;
    }
    if (i == 0) return 8. / 27.;
    if (i <= 6) return 2. / 27.;
    if (i <= 18) return 1. / 54.;
    return 1. / 216.;
}

static void feq_bgk(int q, double rho, const double *u, double *feq)
{
    double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    for (int i = 0; i < q; ++i) {
        double euv = EX[i] * u[0] + EY[i] * u[1] + EZ[i] * u[2];
        feq[i] = rho * wq(q, i) * (1. + 3. * euv + 4.5 * euv * euv - 1.5 * uu);
    }
}

static double feq_bgk_one(int q, double rho, const double *u, int i)
{
    double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    double euv = EX[i] * u[0] + EY[i] * u[1] + EZ[i] * u[2];
    return rho * wq(q, i) * (1. + 3. * euv + 4.5 * euv * euv - 1.5 * uu);
}

static void feq_heluo(int q, double rho, const double *u, double *feq)
{
    double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    for (int i = 0; i < q; ++i) {
        double euv = EX[i] * u[0] + EY[i] * u[1] + EZ[i] * u[2];
        feq[i] = wq(q, i) * (rho + 1.0 * (3. * euv + 4.5 * euv * euv - 1.5 * uu));
    }
}

static void macros_of(int q, const double *d, double *rho, double *u)
{
    double r = d[0], vx = 0., vy = 0., vz = 0.;
    for (int i = 1; i < q; ++i) {
        r += d[i];
        vx += d[i] * EX[i];
        vy += d[i] * EY[i];
        vz += d[i] * EZ[i];
    }
    double s = (r > -1e-6 && r < 1e-6) ? ((r < 0.0) ? -1e-6 : 1e-6) : r;
    *rho = r;
    u[0] = vx / s;
    u[1] = vy / s;
    u[2] = vz / s;
}

/* ------------------------------------------------------------------ */
/* D3Q27 cumulant collision (Collision_Cumulant.cpp:320-652): central    */
/* moments, cumulants with rho floor, relaxation (omega1 = 1/tau, bulk   */
/* omega2 = 1, all cumulants of order >= 3 set to zero), inverse.        */
/* ------------------------------------------------------------------ */
/* central-moment slots: index = a + 3b + 9c holds the (a,b,c) moment */
#define M(a, b, c) m[(a) + 3 * (b) + 9 * (c)]

static double safe_irho(double r)
{
    return 1.0 / ((r > -1e-6 && r < 1e-6) ? ((r < 0.0) ? -1e-6 : 1e-6) : r);
}

/* backward chimera step along one axis: moments (a0,a1,a2) of orders
 * 0,1,2 in that axis -> populations at offsets -1, 0, +1 */
static void chim_back(double a0, double a1, double a2, double v, double v2, double *pn, double *pz, double *pp)
{
    *pz = a0 * (1 - v2) - a1 * 2 * v - a2;
    *pn = (a0 * (v2 - v) + a1 * (2 * v - 1) + a2) * 0.5;
    *pp = (a0 * (v2 + v) + a1 * (2 * v + 1) + a2) * 0.5;
}

static void cumulant_collide(const double *f, double rho, const double *u, double tau, double *out)
{
    double m[27];
    for (int i = 0; i < 27; ++i) m[i] = 0.;
    for (int i = 0; i < 27; ++i) {
        double cx = EX[i] - u[0], cy = EY[i] - u[1], cz = EZ[i] - u[2], fi = f[i];
        M(0, 0, 0) += fi;
        M(1, 0, 0) += cx * fi;
        M(0, 1, 0) += cy * fi;
        M(0, 0, 1) += cz * fi;
        M(2, 0, 0) += cx * cx * fi;
        M(0, 2, 0) += cy * cy * fi;
        M(0, 0, 2) += cz * cz * fi;
        M(1, 1, 0) += cx * cy * fi;
        M(1, 0, 1) += cx * cz * fi;
        M(0, 1, 1) += cy * cz * fi;
        M(2, 1, 0) += cx * cx * cy * fi;
        M(2, 0, 1) += cx * cx * cz * fi;
        M(0, 2, 1) += cy * cy * cz * fi;
        M(1, 2, 0) += cx * cy * cy * fi;
        M(1, 0, 2) += cx * cz * cz * fi;
        M(0, 1, 2) += cy * cz * cz * fi;
        M(1, 1, 1) += cx * cy * cz * fi;
        M(2, 2, 0) += cx * cx * cy * cy * fi;
        M(2, 0, 2) += cx * cx * cz * cz * fi;
        M(0, 2, 2) += cy * cy * cz * cz * fi;
        M(2, 1, 1) += cx * cx * cy * cz * fi;
        M(1, 2, 1) += cx * cy * cy * cz * fi;
        M(1, 1, 2) += cx * cy * cz * cz * fi;
        M(2, 2, 1) += cx * cx * cy * cy * cz * fi;
        M(2, 1, 2) += cx * cx * cy * cz * cz * fi;
        M(1, 2, 2) += cx * cy * cy * cz * cz * fi;
        M(2, 2, 2) += cx * cx * cy * cy * cz * cz * fi;
    }
    /* second-order cumulants equal the central moments; only they survive
     * the relaxation (higher orders are reset to zero below) */
    double c200 = M(2, 0, 0), c020 = M(0, 2, 0), c002 = M(0, 0, 2);
    double c110 = M(1, 1, 0), c101 = M(1, 0, 1), c011 = M(0, 1, 1);
    double k000 = M(0, 0, 0);
    double om1 = 1. / tau, om2 = 1.;
    double irho = safe_irho(rho);
    double dxu = -(om1 * (2 * c200 - c020 - c002) + om2 * (c200 + c020 + c002 - k000)) * irho * 0.5;
    double dyv = dxu + 3 * om1 * (c200 - c020) * 0.5 * irho;
    double dzw = dxu + 3 * om1 * (c200 - c002) * 0.5 * irho;
    c110 *= (1 - om1);
    c101 *= (1 - om1);
    c011 *= (1 - om1);
    double ux2 = ((u[0]) * (u[0])), uy2 = ((u[1]) * (u[1])), uz2 = ((u[2]) * (u[2]));
    double x1 = (1 - om1) * (c200 - c020) - 3 * rho * (1 - om1 * 0.5) * (ux2 * dxu - uy2 * dyv);
    double x2 = (1 - om1) * (c200 - c002) - 3 * rho * (1 - om1 * 0.5) * (ux2 * dxu - uz2 * dzw);
    double x3 = k000 * om2 + (1 - om2) * (c200 + c020 + c002) -
                3 * rho * (1 - om2 * 0.5) * (ux2 * dxu + uy2 * dyv + uz2 * dzw);
    c200 = (x1 + x2 + x3) / 3;
    c020 = c200 - x1;
    c002 = c200 - x2;

    /* back to central moments (orders 0 and 1 keep their forward values) */
    double k[27];
    for (int i = 0; i < 27; ++i) k[i] = m[i];
    double ir = safe_irho(rho);
#define K(a, b, cc) k[(a) + 3 * (b) + 9 * (cc)]
    K(1, 1, 0) = c110; K(0, 1, 1) = c011; K(1, 0, 1) = c101;
    K(2, 0, 0) = c200; K(0, 2, 0) = c020; K(0, 0, 2) = c002;
    /* the relaxed third-order cumulants are zero; the (2,1,0), (1,0,2) and
     * (0,2,1) moments are not reassigned by the reference's backward
     * transform (Collision_Cumulant.cpp:451-454) and keep their forward
     * central-moment values */
    K(1, 2, 0) = 0; K(0, 1, 2) = 0; K(2, 0, 1) = 0;
    K(1, 1, 1) = 0;
    K(2, 1, 1) = 0 + (K(2, 0, 0) * K(0, 1, 1) + 2 * K(1, 1, 0) * K(1, 0, 1)) * ir;
    K(1, 2, 1) = 0 + (K(0, 2, 0) * K(1, 0, 1) + 2 * K(0, 1, 1) * K(1, 1, 0)) * ir;
    K(1, 1, 2) = 0 + (K(0, 0, 2) * K(1, 1, 0) + 2 * K(1, 0, 1) * K(0, 1, 1)) * ir;
    K(2, 2, 0) = 0 + (K(2, 0, 0) * K(0, 2, 0) + 2 * K(1, 1, 0) * K(1, 1, 0)) * ir;
    K(0, 2, 2) = 0 + (K(0, 2, 0) * K(0, 0, 2) + 2 * K(0, 1, 1) * K(0, 1, 1)) * ir;
    K(2, 0, 2) = 0 + (K(0, 0, 2) * K(2, 0, 0) + 2 * K(1, 0, 1) * K(1, 0, 1)) * ir;
    K(1, 2, 2) = 0 + (K(0, 0, 2) * K(1, 2, 0) + K(0, 2, 0) * K(1, 0, 2) + 4 * K(0, 1, 1) * K(1, 1, 1) +
                      2 * (K(1, 0, 1) * K(0, 2, 1) + K(1, 1, 0) * K(0, 1, 2))) * ir;
    K(2, 1, 2) = 0 + (K(2, 0, 0) * K(0, 1, 2) + K(0, 0, 2) * K(2, 1, 0) + 4 * K(1, 0, 1) * K(1, 1, 1) +
                      2 * (K(1, 1, 0) * K(1, 0, 2) + K(0, 1, 1) * K(2, 0, 1))) * ir;
    K(2, 2, 1) = 0 + (K(0, 2, 0) * K(2, 0, 1) + K(2, 0, 0) * K(0, 2, 1) + 4 * K(1, 1, 0) * K(1, 1, 1) +
                      2 * (K(0, 1, 1) * K(2, 1, 0) + K(1, 0, 1) * K(1, 2, 0))) * ir;
    {
        double a = (4 * K(1, 1, 1) * K(1, 1, 1) + K(2, 0, 0) * K(0, 2, 2) + K(0, 2, 0) * K(2, 0, 2) +
                    K(0, 0, 2) * K(2, 2, 0) + 4 * (K(0, 1, 1) * K(2, 1, 1) + K(1, 0, 1) * K(1, 2, 1) + K(1, 1, 0) * K(1, 1, 2)) +
                    2 * (K(1, 2, 0) * K(1, 0, 2) + K(2, 1, 0) * K(0, 1, 2) + K(2, 0, 1) * K(0, 2, 1))) * ir;
        double b = (16 * K(1, 1, 0) * K(1, 0, 1) * K(0, 1, 1) +
                    4 * (K(1, 0, 1) * K(1, 0, 1) * K(0, 2, 0) + K(0, 1, 1) * K(0, 1, 1) * K(2, 0, 0) + K(1, 1, 0) * K(1, 1, 0) * K(0, 0, 2)) +
                    2 * K(2, 0, 0) * K(0, 2, 0) * K(0, 0, 2)) * ir * ir;
        K(2, 2, 2) = 0 + a - b;
    }
    /* backward chimera: x pass, then y, then z */
    double ux = u[0], uy = u[1], uz = u[2];
    double ux2b = ((ux) * (ux)), uy2b = ((uy) * (uy)), uz2b = ((uz) * (uz));
    double p1[27], p2[27], p3[27]; /* p1[(ix) + 3 b + 9 c], ix in {-1,0,+1} -> 0,1,2 */
    for (int cc = 0; cc < 3; ++cc)
        for (int b = 0; b < 3; ++b)
            chim_back(K(0, b, cc), K(1, b, cc), K(2, b, cc), ux, ux2b, &p1[0 + 3 * b + 9 * cc],
                      &p1[1 + 3 * b + 9 * cc], &p1[2 + 3 * b + 9 * cc]);
    for (int ix = 0; ix < 3; ++ix)
        for (int cc = 0; cc < 3; ++cc)
            chim_back(p1[ix + 0 + 9 * cc], p1[ix + 3 + 9 * cc], p1[ix + 6 + 9 * cc], uy, uy2b,
                      &p2[ix + 0 + 9 * cc], &p2[ix + 3 + 9 * cc], &p2[ix + 6 + 9 * cc]);
    for (int ix = 0; ix < 3; ++ix)
        for (int iy = 0; iy < 3; ++iy)
            chim_back(p2[ix + 3 * iy + 0], p2[ix + 3 * iy + 9], p2[ix + 3 * iy + 18], uz, uz2b,
                      &p3[ix + 3 * iy + 0], &p3[ix + 3 * iy + 9], &p3[ix + 3 * iy + 18]);
    /* slot (sx,sy,sz) with s = 0 for -1, 1 for 0, 2 for +1 */
    for (int i = 0; i < 27; ++i) out[i] = p3[(EX[i] + 1) + 3 * (EY[i] + 1) + 9 * (EZ[i] + 1)];
#undef K
}
#undef M

/* ------------------------------------------------------------------ */
/* Case construction                                                  */
/* ------------------------------------------------------------------ */
static void kv_push(keyvec *v, const uint64_t *k, int64_t n)
{
    if (v->n + n > v->cap) {
        int64_t nc = (v->n + n) * 2 + 16;
        v->keys = (uint64_t *)realloc(v->keys, (size_t)nc * sizeof(uint64_t));
        v->cap = nc;
    }
    memcpy(v->keys + v->n, k, (size_t)n * sizeof(uint64_t));
    v->n += n;
}

static int cmp_u64(const void *a, const void *b)
{
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

static int64_t sort_unique(uint64_t *k, int64_t n)
{
    if (n == 0) return 0;
    qsort(k, (size_t)n, sizeof(uint64_t), cmp_u64);
    int64_t m = 1;
    for (int64_t i = 1; i < n; ++i)
        if (k[i] != k[m - 1]) k[m++] = k[i];
    return m;
}

void *oc_case_new(int q, int max_level, int collision, int ib_method, int bc_mode, int stream_conv,
                  const int *periodic, const int64_t *extent0, const double *tau, double rho0,
                  const double *u_bc)
{
    if ((q != 19 && q != 27) || max_level < 0 || max_level >= OC_MAXL) return NULL;
    if (collision == COLL_CUMULANT && q != 27) return NULL;
    if (bc_mode == BC_ZOUHE_HH && (q != 19 || collision != COLL_LBGK)) return NULL;
    oc_case *c = (oc_case *)calloc(1, sizeof(oc_case));
    c->q = q;
    c->L = max_level;
    c->collision = collision;
    c->ib_method = ib_method;
    c->bc_mode = bc_mode;
    c->stream_conv = stream_conv;
    for (int a = 0; a < 3; ++a) {
        c->periodic[a] = periodic[a];
        c->extent0[a] = extent0[a];
        c->u_bc[a] = u_bc[a];
        for (int f = 0; f < 6; ++f) c->face_u[f][a] = u_bc[a];
    }
    for (int l = 0; l <= max_level; ++l) c->tau[l] = tau[l];
    c->rho0 = rho0;
    return c;
}

void oc_case_free(void *h)
{
    oc_case *c = (oc_case *)h;
    if (!c) return;
    for (int l = 0; l <= c->L; ++l) {
        oc_level *lv = &c->lv[l];
        free(lv->key); free(lv->tag); free(lv->bcidx); free(lv->disrow);
        free(lv->f); free(lv->fcol); free(lv->rho); free(lv->u);
        for (int s = 0; s < OC_NSETS; ++s) { free(lv->list[s]); free(lv->raw[s].keys); }
        for (int b = 0; b < 26; ++b) { free(lv->bclist[b]); free(lv->rawbc[b].keys); }
        free(lv->band); free(lv->rawband.keys); free(lv->prev);
    }
    free(c->dis_key); free(c->dis);
    free(c->mref); free(c->mdv); free(c->path); free(c->acc);
    free(c);
}

int oc_add_set(void *h, int level, int set_id, const uint64_t *keys, int64_t n)
{
    oc_case *c = (oc_case *)h;
    if (level < 0 || level > c->L || c->built) return -1;
    if (set_id >= S_BC0 && set_id < S_BC0 + 26) {
        if (level != 0) return -1;
        kv_push(&c->lv[0].rawbc[set_id - S_BC0], keys, n);
        return 0;
    }
    if (set_id == S_BAND) {
        if (level != c->L) return -1;
        kv_push(&c->lv[level].rawband, keys, n);
        return 0;
    }
    if (set_id < 0 || set_id >= OC_NSETS) return -1;
    kv_push(&c->lv[level].raw[set_id], keys, n);
    return 0;
}

int oc_set_dis(void *h, const uint64_t *keys, const double *rows, int64_t n)
{
    oc_case *c = (oc_case *)h;
    int w = c->q - 1;
    c->ndis = n;
    c->dis_key = (uint64_t *)malloc((size_t)(n ? n : 1) * sizeof(uint64_t));
    c->dis = (double *)malloc((size_t)(n ? n : 1) * (size_t)w * sizeof(double));
    memcpy(c->dis_key, keys, (size_t)n * sizeof(uint64_t));
    memcpy(c->dis, rows, (size_t)n * (size_t)w * sizeof(double));
    for (int64_t i = 1; i < n; ++i)
        if (keys[i] <= keys[i - 1]) return -1; /* rows must come sorted by key */
    return 0;
}

static int64_t *index_list(oc_level *lv, keyvec *kv, int64_t *nout, uint32_t tagbit)
{
    int64_t m = sort_unique(kv->keys, kv->n);
    int64_t *out = (int64_t *)malloc((size_t)(m ? m : 1) * sizeof(int64_t));
    for (int64_t i = 0; i < m; ++i) {
        out[i] = find_idx(lv, kv->keys[i]);
        lv->tag[out[i]] |= tagbit;
    }
    *nout = m;
    return out;
}

int oc_build(void *h)
{
    oc_case *c = (oc_case *)h;
    int q = c->q;
    for (int l = 0; l <= c->L; ++l) {
        oc_level *lv = &c->lv[l];
        int64_t tot = 0;
        for (int s = 0; s < OC_NSETS; ++s) tot += lv->raw[s].n;
        for (int b = 0; b < 26; ++b) tot += lv->rawbc[b].n;
        uint64_t *all = (uint64_t *)malloc((size_t)(tot ? tot : 1) * sizeof(uint64_t));
        int64_t p = 0;
        for (int s = 0; s < OC_NSETS; ++s) { memcpy(all + p, lv->raw[s].keys, (size_t)lv->raw[s].n * 8); p += lv->raw[s].n; }
        for (int b = 0; b < 26; ++b) { memcpy(all + p, lv->rawbc[b].keys, (size_t)lv->rawbc[b].n * 8); p += lv->rawbc[b].n; }
        lv->n = sort_unique(all, tot);
        lv->key = all;
        int64_t n = lv->n ? lv->n : 1;
        lv->tag = (uint32_t *)calloc((size_t)n, sizeof(uint32_t));
        lv->bcidx = (int8_t *)malloc((size_t)n);
        memset(lv->bcidx, -1, (size_t)n);
        lv->disrow = (int32_t *)malloc((size_t)n * sizeof(int32_t));
        for (int64_t i = 0; i < n; ++i) lv->disrow[i] = -1;
        static const uint32_t bits[OC_NSETS] = {T_LATF, T_F2C, T_C2F, T_GC2F, T_GF2C, T_SF};
        for (int s = 0; s < OC_NSETS; ++s) lv->list[s] = index_list(lv, &lv->raw[s], &lv->nlist[s], bits[s]);
        for (int b = 0; b < 26; ++b) {
            lv->bclist[b] = index_list(lv, &lv->rawbc[b], &lv->nbc[b], T_BC);
            for (int64_t i = 0; i < lv->nbc[b]; ++i) lv->bcidx[lv->bclist[b][i]] = (int8_t)b;
        }
        lv->f = (double *)calloc((size_t)n * (size_t)q, sizeof(double));
        lv->fcol = (double *)calloc((size_t)n * (size_t)q, sizeof(double));
        lv->rho = (double *)calloc((size_t)n, sizeof(double));
        lv->u = (double *)calloc((size_t)n * 3, sizeof(double));
    }
    oc_level *fl = &c->lv[c->L];
    fl->band = index_list(fl, &fl->rawband, &fl->nband, T_BAND);
    if (fl->nband) c->acc = (int64_t *)calloc((size_t)fl->n * 3, sizeof(int64_t));
    for (int64_t r = 0; r < c->ndis; ++r) {
        int64_t i = find_idx(fl, c->dis_key[r]);
        if (i < 0) return -2;
        fl->disrow[i] = (int32_t)r;
        fl->tag[i] |= T_IB;
    }
    c->built = 1;
    return 0;
}

/* Reference initial state (LBM_Manager.cpp:482-592, 296-304): every stored
 * cell gets f = fcol = feq(rho0, u0) and rho = rho0, u = u0; finest-level
 * solid cells get f = fcol = 0 and rho = 1. */
int oc_init_equilibrium(void *h, double rho0, const double *u0)
{
    oc_case *c = (oc_case *)h;
    c->prev_stale = 1;
    int q = c->q;
    double feq[27];
    feq_bgk(q, rho0, u0, feq);
    for (int l = 0; l <= c->L; ++l) {
        oc_level *lv = &c->lv[l];
        for (int64_t i = 0; i < lv->n; ++i) {
            int solid = (lv->tag[i] & T_SF) && !(lv->tag[i] & (T_LATF | T_F2C | T_C2F | T_GC2F | T_BC));
            for (int k = 0; k < q; ++k) {
                lv->f[k * lv->n + i] = solid ? 0. : feq[k];
                lv->fcol[k * lv->n + i] = solid ? 0. : feq[k];
            }
            lv->rho[i] = solid ? 1. : rho0;
            for (int a = 0; a < 3; ++a) lv->u[3 * i + a] = solid ? 0. : u0[a];
        }
    }
    return 0;
}

int64_t oc_level_size(void *h, int level) { return ((oc_case *)h)->lv[level].n; }

int oc_get_level(void *h, int level, uint64_t *keys, uint32_t *tags, double *f, double *fcol, double *rho,
                 double *u)
{
    oc_case *c = (oc_case *)h;
    oc_level *lv = &c->lv[level];
    size_t n = (size_t)lv->n;
    if (keys) memcpy(keys, lv->key, n * 8);
    if (tags) memcpy(tags, lv->tag, n * 4);
    if (f) memcpy(f, lv->f, n * (size_t)c->q * 8);
    if (fcol) memcpy(fcol, lv->fcol, n * (size_t)c->q * 8);
    if (rho) memcpy(rho, lv->rho, n * 8);
    if (u) memcpy(u, lv->u, n * 24);
    return 0;
}

int oc_set_level(void *h, int level, const double *f, const double *fcol, const double *rho, const double *u)
{
    oc_case *c = (oc_case *)h;
    oc_level *lv = &c->lv[level];
    size_t n = (size_t)lv->n;
    if (f) memcpy(lv->f, f, n * (size_t)c->q * 8);
    if (fcol) memcpy(lv->fcol, fcol, n * (size_t)c->q * 8);
    if (rho) memcpy(lv->rho, rho, n * 8);
    if (u) memcpy(lv->u, u, n * 24);
    c->prev_stale = 1;
    return 0;
}

void oc_get_force(void *h, double *out)
{
    oc_case *c = (oc_case *)h;
    out[0] = c->fx; out[1] = c->fy; out[2] = c->fz; out[3] = (double)c->nforce;
}

void oc_reset_force(void *h)
{
    oc_case *c = (oc_case *)h;
    c->fx = c->fy = c->fz = 0.;
    c->nforce = 0;
}

/* neighbour index of cell i along q, following the configured pull
 * convention: the reference pulls from x + e_q (Stream_Manager.cpp:53,62);
 * the textbook convention pulls from x - e_q */
static int64_t pull_src(const oc_case *c, const oc_level *lv, int level, int64_t i, int k)
{
    int s = c->stream_conv ? -1 : 1;
    uint64_t nk = find_neighbor(c, lv->key[i], level, s * EX[k], s * EY[k], s * EZ[k]);
    return find_idx(lv, nk);
}

/* ------------------------------------------------------------------ */
/* Per-phase operations                                                */
/* ------------------------------------------------------------------ */
/* LBM_Manager::calculateMacros(level) (LBM_Manager.cpp:1003-1050) */
static void phase_macros(oc_case *c, int l)
{
    oc_level *lv = &c->lv[l];
    int q = c->q;
    double d[27];
    for (int s = 0; s < 2; ++s) {
        int64_t nl = lv->nlist[s == 0 ? S_LATF : S_F2C];
        int64_t *li = lv->list[s == 0 ? S_LATF : S_F2C];
        for (int64_t j = 0; j < nl; ++j) {
            int64_t i = li[j];
            for (int k = 0; k < q; ++k) d[k] = lv->f[k * lv->n + i];
            macros_of(q, d, &lv->rho[i], &lv->u[3 * i]);
        }
    }
}

/* Collision_LBGK::collide / Collision_Cumulant::collide
 * (Collision_Manager.cpp:13-53, Collision_Cumulant.cpp:22-159) */
static void band_collide(oc_case *c, int l, int64_t i);

static void phase_collide(oc_case *c, int l)
{
    oc_level *lv = &c->lv[l];
    int q = c->q;
    double tau0 = c->tau[l];
    double feq[27], d[27], o[27];
    for (int s = 0; s < 2; ++s) {
        int64_t nl = lv->nlist[s == 0 ? S_LATF : S_F2C];
        int64_t *li = lv->list[s == 0 ? S_LATF : S_F2C];
        for (int64_t j = 0; j < nl; ++j) {
            int64_t i = li[j];
            if (lv->tag[i] & T_BAND) {
                band_collide(c, l, i);
                continue;
            }
            if (c->collision == COLL_LBGK) {
                feq_bgk(q, lv->rho[i], &lv->u[3 * i], feq);
                for (int k = 0; k < q; ++k) {
                    double fk = lv->f[k * lv->n + i];
                    lv->fcol[k * lv->n + i] = fk - (fk - feq[k]) / tau0;
                }
            } else {
                for (int k = 0; k < 27; ++k) d[k] = lv->f[k * lv->n + i];
                cumulant_collide(d, lv->rho[i], &lv->u[3 * i], tau0, o);
                for (int k = 0; k < 27; ++k) lv->fcol[k * lv->n + i] = o[k];
            }
        }
    }
    for (int64_t j = 0; j < lv->nlist[S_C2F]; ++j) {
        int64_t i = lv->list[S_C2F][j];
        for (int k = 0; k < q; ++k) lv->fcol[k * lv->n + i] = lv->f[k * lv->n + i];
    }
}

/* ABPatternPull::stream (Stream_Manager.cpp:43-76): a missing neighbour
 * keeps the previous f */
static void phase_stream(oc_case *c, int l)
{
    oc_level *lv = &c->lv[l];
    int q = c->q;
    for (int s = 0; s < 2; ++s) {
        int64_t nl = lv->nlist[s == 0 ? S_LATF : S_C2F];
        int64_t *li = lv->list[s == 0 ? S_LATF : S_C2F];
        for (int64_t j = 0; j < nl; ++j) {
            int64_t i = li[j];
            lv->f[i] = lv->fcol[i];
            for (int k = 1; k < q; ++k) {
                int64_t src = pull_src(c, lv, l, i, k);
                if (src < 0) continue;
                lv->f[k * lv->n + i] = lv->fcol[k * lv->n + src];
            }
        }
    }
}

static void children_of(const oc_case *c, uint64_t code, int fine, uint64_t *ch)
{
    /* child order (0,0,0),(1,0,0),(0,1,0),(1,1,0),(0,0,1),(1,0,1),(0,1,1),(1,1,1)
     * -- the reference's find_x1/find_y1/find_z1 composition
     * (LBM_Manager.cpp:1074-1082) */
    uint64_t x1 = find_neighbor(c, code, fine, 1, 0, 0);
    uint64_t y1 = find_neighbor(c, code, fine, 0, 1, 0);
    uint64_t xy1 = find_neighbor(c, x1, fine, 0, 1, 0);
    ch[0] = code;
    ch[1] = x1;
    ch[2] = y1;
    ch[3] = xy1;
    ch[4] = find_neighbor(c, code, fine, 0, 0, 1);
    ch[5] = find_neighbor(c, x1, fine, 0, 0, 1);
    ch[6] = find_neighbor(c, y1, fine, 0, 0, 1);
    ch[7] = find_neighbor(c, xy1, fine, 0, 0, 1);
}

/* LBM_Manager::AMR_transDDF_explosion (LBM_Manager.cpp:1059-1129) */
/* the explosion sources of level `fine` (F2C then ghost F2C of its parent)
 * as one list: source s -> parent cell index */
static int64_t expl_source(const oc_level *cl, int64_t s)
{
    return s < cl->nlist[S_F2C] ? cl->list[S_F2C][s] : cl->list[S_GF2C][s - cl->nlist[S_F2C]];
}

/* parent values of every source into fl->prev [q][nsources] */
static void save_sources(oc_case *c, int fine)
{
    oc_level *cl = &c->lv[fine - 1], *fl = &c->lv[fine];
    int64_t ns = cl->nlist[S_F2C] + cl->nlist[S_GF2C];
    if (!fl->prev) fl->prev = (double *)calloc((size_t)(c->q * ns + 1), sizeof(double));
    for (int64_t s = 0; s < ns; ++s) {
        int64_t i = expl_source(cl, s);
        for (int k = 0; k < c->q; ++k) fl->prev[k * ns + s] = cl->fcol[k * cl->n + i];
    }
}

static int phase_explosion(oc_case *c, int fine, int extrap)
{
    int coarse = fine - 1, q = c->q;
    oc_level *cl = &c->lv[coarse], *fl = &c->lv[fine];
    double scale = (2.0 * c->tau[fine]) / c->tau[coarse];
    double dc[27], feq[27], rho, u[3];
    uint64_t ch[8];
    const int64_t ns = cl->nlist[S_F2C] + cl->nlist[S_GF2C];
    for (int pass = 0; pass < 2; ++pass) {
        int64_t nl = cl->nlist[pass == 0 ? S_F2C : S_GF2C];
        int64_t *li = cl->list[pass == 0 ? S_F2C : S_GF2C];
        for (int64_t j = 0; j < nl; ++j) {
            int64_t i = li[j];
            const int64_t sidx = pass == 0 ? j : cl->nlist[S_F2C] + j;
            for (int k = 0; k < q; ++k) dc[k] = cl->fcol[k * cl->n + i];
            if (extrap)
                for (int k = 0; k < q; ++k) dc[k] = 1.5 * dc[k] - 0.5 * fl->prev[k * ns + sidx];
            macros_of(q, dc, &rho, u);
            feq_heluo(q, rho, u, feq);
            children_of(c, cl->key[i], fine, ch);
            for (int m = 0; m < 8; ++m) {
                int64_t fi = find_idx(fl, ch[m]);
                /* the skip test looks the raw key up in dis, whatever level
                 * the key belongs to (LBM_Manager.cpp:1095,1121) */
                if (find_sorted(c->dis_key, c->ndis, ch[m]) >= 0) continue;
                if (pass == 1 && (fi < 0 || !(fl->tag[fi] & T_GC2F))) continue;
                if (fi < 0) return -3; /* .at() would throw */
                for (int k = 0; k < q; ++k) fl->fcol[k * fl->n + fi] = feq[k] + scale * (dc[k] - feq[k]);
            }
        }
    }
    if (extrap) save_sources(c, fine);
    return 0;
}

/* LBM_Manager::AMR_transDDF_coalescence (LBM_Manager.cpp:1131-1169) */
static int phase_coalescence(oc_case *c, int coarse)
{
    int fine = coarse + 1, q = c->q;
    oc_level *cl = &c->lv[coarse], *fl = &c->lv[fine];
    double scale = c->tau[coarse] / (2.0 * c->tau[fine]);
    double avg[27], feq[27], rho, u[3];
    uint64_t ch[8];
    int64_t fi[8];
    for (int64_t j = 0; j < cl->nlist[S_F2C]; ++j) {
        int64_t i = cl->list[S_F2C][j];
        children_of(c, cl->key[i], fine, ch);
        for (int m = 0; m < 8; ++m) {
            fi[m] = find_idx(fl, ch[m]);
            if (fi[m] < 0) return -4;
        }
        for (int k = 0; k < q; ++k) {
            avg[k] = 0;
            for (int m = 0; m < 8; ++m) avg[k] += fl->f[k * fl->n + fi[m]];
            avg[k] /= 8.0;
        }
        macros_of(q, avg, &rho, u);
        feq_heluo(q, rho, u, feq);
        for (int k = 0; k < q; ++k) cl->f[k * cl->n + i] = feq[k] + scale * (avg[k] - feq[k]);
    }
    return 0;
}

/* non-equilibrium extrapolation, "eflow stable" form
 * (NonEquilibrumExtrapolation.cpp:33-71 and its five siblings), level 0
 * after streaming.  It rewrites only boundary-cell f, which no fluid cell
 * reads, so its in-place update order is immaterial to the flow. */
static int phase_bc_neq(oc_case *c)
{
    oc_level *lv = &c->lv[0];
    int q = c->q, w = (q == 19) ? 14 : 18;
    for (int face = 0; face < 6; ++face) {
        for (int g = 0; g < 9; ++g) {
            int b = FACE_SETS[face][g];
            if (b < 0) break;
            for (int64_t j = 0; j < lv->nbc[b]; ++j) {
                int64_t i = lv->bclist[b][j];
                for (int t = 0; t < w; ++t) {
                    int k = (q == 19) ? BDRY19[b][t] : BDRY27[b][t];
                    if (k < 0) break;
                    uint64_t nk = find_neighbor(c, lv->key[i], 0, EX[k], EY[k], EZ[k]);
                    int64_t nb = find_idx(lv, nk);
                    if (nb < 0) return -5;
                    double fw = feq_bgk_one(q, lv->rho[i], c->face_u[face], k);
                    double fn = feq_bgk_one(q, lv->rho[nb], &lv->u[3 * nb], k);
                    lv->f[k * lv->n + i] = fw + lv->f[k * lv->n + nb] - fn;
                }
            }
        }
    }
    return 0;
}

/* ---- direct forcing on Lagrangian markers (no reference counterpart) ----
 * Restated from Uhlmann (2005) and Roma, Peskin & Berger (1999): the 3-point
 * kernel, marker force 2 rho (U - u) from the interpolated unforced
 * velocity, spreading into int64 fixed point (2^-32), Guo forcing in the
 * collision of the band cells.  Same expression order as the device code. */
#define OC_FSCALE 4294967296.0

static double roma3(double r)
{
    r = fabs(r);
    if (r <= 0.5) return (1.0 + sqrt(1.0 - 3.0 * r * r)) / 3.0;
    if (r <= 1.5) {
        double a = 1.0 - r;
        return (5.0 - 3.0 * r - sqrt(1.0 - 3.0 * a * a)) / 6.0;
    }
    return 0.0;
}

static void band_collide(oc_case *c, int l, int64_t i)
{
    oc_level *lv = &c->lv[l];
    int q = c->q;
    int64_t n = lv->n;
    double d[27], r = 0., jx = 0., jy = 0., jz = 0.;
    for (int k = 0; k < q; ++k) {
        d[k] = lv->f[k * n + i];
        r += d[k];
        jx += d[k] * EX[k];
        jy += d[k] * EY[k];
        jz += d[k] * EZ[k];
    }
    double gx = (double)c->acc[i] / OC_FSCALE, gy = (double)c->acc[n + i] / OC_FSCALE,
           gz = (double)c->acc[2 * n + i] / OC_FSCALE;
    double rs = (r > -1e-6 && r < 1e-6) ? ((r < 0.) ? -1e-6 : 1e-6) : r;
    double x = (jx + gx * 0.5) / rs, y = (jy + gy * 0.5) / rs, z = (jz + gz * 0.5) / rs;
    double om = 1.0 / c->tau[l];
    double fpre = 1.0 - 0.5 * om;
    double uu = x * x + y * y + z * z;
    for (int k = 0; k < q; ++k) {
        double eu = EX[k] * x + EY[k] * y + EZ[k] * z;
        double wk = wq(q, k);
        double feq = r * wk * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uu);
        double ge = (3.0 * (EX[k] - x) + 9.0 * eu * EX[k]) * gx + (3.0 * (EY[k] - y) + 9.0 * eu * EY[k]) * gy +
                    (3.0 * (EZ[k] - z) + 9.0 * eu * EZ[k]) * gz;
        lv->fcol[k * n + i] = d[k] - (d[k] - feq) * om + fpre * wk * ge;
    }
}

static void phase_df(oc_case *c)
{
    int L = c->L, q = c->q;
    oc_level *lv = &c->lv[L];
    int64_t n = lv->n;
    double d[27];
    for (int64_t j = 0; j < lv->nband; ++j) {
        int64_t i = lv->band[j];
        for (int k = 0; k < q; ++k) d[k] = lv->f[k * n + i];
        macros_of(q, d, &lv->rho[i], &lv->u[3 * i]);
        c->acc[i] = 0;
        c->acc[n + i] = 0;
        c->acc[2 * n + i] = 0;
    }
    if (!c->nm) {
        c->nforce += 1;
        return;
    }
    const double *pp = c->path + 6 * (c->tstep % c->period);
    double sx = 0., sy = 0., sz = 0.;
    for (int64_t m = 0; m < c->nm; ++m) {
        double X = c->center[0] + pp[0] + c->mref[m];
        double Y = c->center[1] + pp[1] + c->mref[c->nm + m];
        double Z = c->center[2] + pp[2] + c->mref[2 * c->nm + m];
        int64_t ix = (int64_t)floor(X), iy = (int64_t)floor(Y), iz = (int64_t)floor(Z);
        int64_t idx[27];
        double wgt[27], r = 0., vx = 0., vy = 0., vz = 0.;
        for (int cc = 0; cc < 27; ++cc) {
            int64_t x = ix + cc % 3 - 1, y = iy + (cc / 3) % 3 - 1, z = iz + cc / 9 - 1;
            double wv = roma3((double)x + 0.5 - X) * roma3((double)y + 0.5 - Y) * roma3((double)z + 0.5 - Z);
            int64_t i = -1;
            if (x >= 0 && y >= 0 && z >= 0) {
                uint64_t k = dilate3((uint64_t)x) | (dilate3((uint64_t)y) << 1) | (dilate3((uint64_t)z) << 2);
                i = find_idx(lv, k);
                if (i >= 0 && !(lv->tag[i] & T_BAND)) i = -1;
            }
            idx[cc] = i;
            wgt[cc] = wv;
            if (i >= 0) {
                r += wv * lv->rho[i];
                vx += wv * lv->u[3 * i];
                vy += wv * lv->u[3 * i + 1];
                vz += wv * lv->u[3 * i + 2];
            }
        }
        double fx = 2.0 * r * (pp[3] - vx), fy = 2.0 * r * (pp[4] - vy), fz = 2.0 * r * (pp[5] - vz);
        double dv = c->mdv[m];
        for (int cc = 0; cc < 27; ++cc) {
            int64_t i = idx[cc];
            if (i < 0) continue;
            double sw = wgt[cc] * dv;
            c->acc[i] += (int64_t)llrint(fx * sw * OC_FSCALE);
            c->acc[n + i] += (int64_t)llrint(fy * sw * OC_FSCALE);
            c->acc[2 * n + i] += (int64_t)llrint(fz * sw * OC_FSCALE);
        }
        sx += -fx * dv;
        sy += -fy * dv;
        sz += -fz * dv;
    }
    c->tstep += 1;
    c->fx += sx;
    c->fy += sy;
    c->fz += sz;
    c->nforce += 1;
}

int oc_set_markers(void *h, int64_t nm, const double *ref, const double *dv, const double *center, int64_t period,
                   const double *path)
{
    oc_case *c = (oc_case *)h;
    if (!c->built || !c->acc || period < 1) return -1;
    free(c->mref);
    free(c->mdv);
    free(c->path);
    c->nm = nm;
    c->period = period;
    c->tstep = 0;
    c->mref = (double *)malloc((size_t)(3 * nm + 1) * sizeof(double));
    c->mdv = (double *)malloc((size_t)(nm + 1) * sizeof(double));
    c->path = (double *)malloc((size_t)(6 * period) * sizeof(double));
    memcpy(c->mref, ref, (size_t)(3 * nm) * sizeof(double));
    memcpy(c->mdv, dv, (size_t)nm * sizeof(double));
    memcpy(c->path, path, (size_t)(6 * period) * sizeof(double));
    for (int a = 0; a < 3; ++a) c->center[a] = center[a];
    return 0;
}

/* SinglePointInterpolation::treat (ComplexBoundary_Manager.cpp:43-225):
 * interpolated bounce-back on wall links (Filippova-Haenel or distance
 * weighted), plain pull on free links, density clamp, then eight
 * multi-direct-forcing sweeps on the wall links.  Uses D3Q19 weights for
 * every Q (the remaining D3Q27 weights are zero). */
static void phase_ib(oc_case *c)
{
    if (c->ib_method == IB_DF) {
        phase_df(c);
        return;
    }
    int L = c->L, q = c->q;
    oc_level *lv = &c->lv[L];
    static const double W19[19] = {1. / 3., 1. / 18., 1. / 18., 1. / 18., 1. / 18., 1. / 18., 1. / 18.,
                                   1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36.,
                                   1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36., 1. / 36.};
    double w[27];
    for (int k = 0; k < 27; ++k) w[k] = k < 19 ? W19[k] : 0.;
    double fx = 0., fy = 0., fz = 0.;
    int64_t n = lv->n;
    for (int64_t j = 0; j < lv->nlist[S_LATF]; ++j) {
        int64_t i = lv->list[S_LATF][j];
        if (lv->disrow[i] < 0) continue;
        const double *dr = c->dis + (size_t)lv->disrow[i] * (size_t)(q - 1);
        double rho_b = lv->rho[i];
        lv->f[i] = lv->fcol[i];
        for (int k = 1; k < q; ++k) {
            double d = dr[INV[k] - 1];
            if (d != -1.) {
                double finc = lv->fcol[INV[k] * n + i];
                uint64_t ik = find_neighbor(c, lv->key[i], L, EX[INV[k]], EY[INV[k]], EZ[INV[k]]);
                int64_t si = find_idx(lv, ik);
                double fstr = si >= 0 ? lv->fcol[k * n + si] : finc;
                double fnew;
                if (c->ib_method == IB_FH) {
                    if (d < 0.5) {
                        fnew = (1.0 - 2.0 * d) * finc + 2.0 * d * fstr;
                    } else {
                        double feqw = w[INV[k]] * rho_b;
                        double inv2d = 1.0 / (2.0 * d);
                        fnew = inv2d * fstr + (1.0 - inv2d) * feqw;
                    }
                } else {
                    fnew = (1.0 - d) * finc + d * fstr;
                }
                lv->f[k * n + i] = fnew;
                double mt = finc + fnew;
                fx += -mt * EX[k];
                fy += -mt * EY[k];
                fz += -mt * EZ[k];
            } else {
                uint64_t nk = find_neighbor(c, lv->key[i], L, EX[k], EY[k], EZ[k]);
                int64_t si = find_idx(lv, nk);
                lv->f[k * n + i] = si < 0 ? lv->fcol[INV[k] * n + i] : lv->fcol[k * n + si];
            }
        }
        double ra = 0.;
        for (int k = 0; k < q; ++k) ra += lv->f[k * n + i];
        if (ra < 0.3)
            lv->f[i] += 1.0 * (0.3 - ra);
        else if (ra < 0.5)
            lv->f[i] += 0.5 * (0.5 - ra);
        else if (ra > 3.0)
            lv->f[i] += 1.0 * (3.0 - ra);
        else if (ra > 2.0)
            lv->f[i] += 0.5 * (2.0 - ra);
    }
    c->fx += fx;
    c->fy += fy;
    c->fz += fz;
    c->nforce += 1;
    for (int it = 0; it < 8; ++it) {
        for (int64_t j = 0; j < lv->nlist[S_LATF]; ++j) {
            int64_t i = lv->list[S_LATF][j];
            if (lv->disrow[i] < 0) continue;
            const double *dr = c->dis + (size_t)lv->disrow[i] * (size_t)(q - 1);
            double rho = 0., ux = 0., uy = 0., uz = 0.;
            for (int k = 0; k < q; ++k) {
                double fk = lv->f[k * n + i];
                rho += fk;
                ux += fk * EX[k];
                uy += fk * EY[k];
                uz += fk * EZ[k];
            }
            if (rho <= 0.) continue;
            ux = ux / rho;
            uy = uy / rho;
            uz = uz / rho;
            double um = sqrt(ux * ux + uy * uy + uz * uz);
            if (um < 1e-10) continue;
            double mx = -0.5 * rho * ux, my = -0.5 * rho * uy, mz = -0.5 * rho * uz;
            double adj = 0.;
            for (int k = 1; k < q; ++k) {
                if (dr[INV[k] - 1] == -1.) continue;
                double df = w[k] * 3.0 * (EX[k] * mx + EY[k] * my + EZ[k] * mz);
                lv->f[k * n + i] += df;
                adj -= df;
            }
            lv->f[i] += adj;
        }
    }
}

/* Restated domain boundaries with no runnable reference code: a velocity
 * inlet on the West face and a zero-gradient outflow on the East face, both
 * on boundary-shell cells whose fcol the fluid pulls from.  The inlet keeps
 * fcol = feq(rho0, u_bc) on the wall cell (the West branch of
 * BC/ZouHe_Velocity.cpp:62-115 writes the equilibrium at the boundary cell's
 * own density, which nothing updates from rho0); the outflow copies the inner
 * neighbour's post-collision populations (BC/Outflow.cpp:39-52 copies the
 * populations that stream inward from the first interior layer). */
static int phase_bc_inout(oc_case *c)
{
    oc_level *lv = &c->lv[0];
    int q = c->q;
    double feq[27];
    for (int face = 0; face < 2; ++face) {
        int64_t nl = lv->nbc[face];
        int64_t *li = lv->bclist[face];
        for (int64_t j = 0; j < nl; ++j) {
            int64_t i = li[j];
            uint64_t nk = find_neighbor(c, lv->key[i], 0, face == 0 ? 1 : -1, 0, 0);
            int64_t nb = find_idx(lv, nk);
            if (nb < 0) return -6;
            if (face == 0) {
                feq_bgk(q, c->rho0, c->face_u[0], feq);
                for (int k = 0; k < q; ++k) {
                    lv->fcol[k * lv->n + i] = feq[k];
                    lv->f[k * lv->n + i] = feq[k];
                }
            } else {
                for (int k = 0; k < q; ++k) {
                    lv->fcol[k * lv->n + i] = lv->fcol[k * lv->n + nb];
                    lv->f[k * lv->n + i] = lv->fcol[k * lv->n + nb];
                }
            }
        }
    }
    return 0;
}

/* Restated wet-node boundaries on the x faces (MT_BC_ZOUHE_HH, D3Q19 LBGK;
 * no runnable reference code: BC/ZouHe_Velocity.cpp and BC/Outflow.cpp need
 * the ghost layers that BC_NO_GHOST removes).  After the level-0 stream the
 * boundary-shell cells of the West and East faces pull what their
 * neighbours hold, as fluid cells do (a missing source keeps f), and
 * complete the populations that would come from outside the box:
 *   West: the velocity inlet of BC/ZouHe_Velocity.cpp:170-199 (Zou-He with
 *   the Hecht-Harting transverse corrections; the East formulas there, the
 *   West ones at :81-93): rho from the known populations, the normal one
 *   from its opposite plus rho U_x / 3, the four diagonal ones with the
 *   transverse corrections N_y, N_z;
 *   East: the outflow of BC/Outflow.cpp:39-52, the five incoming populations
 *   copied from the inner neighbour's streamed ones.
 * The formulas are written for a textbook (push-along-e) stream; with the
 * reference's reversed pull they act on g_k = f_inv(k) and the velocity
 * -u_bc (the same scheme mirrored), which keeps the inflow mass balance
 * consistent with the stream direction.  The completed cells then collide
 * (LBGK, level-0 tau) so that the fluid pulls post-collision populations
 * from them as from any other cell. */
static const int HH_IN_E[5] = {2, 8, 10, 12, 14};

static int phase_bc_hh(oc_case *c)
{
    oc_level *lv = &c->lv[0];
    const int64_t n = lv->n;
    const int tb = c->stream_conv != 0;
    const double sgn = tb ? 1.0 : -1.0;
    const double Ux = sgn * c->face_u[0][0], Uy = sgn * c->face_u[0][1], Uz = sgn * c->face_u[0][2];
    for (int face = 0; face < 2; ++face) {
        for (int64_t j = 0; j < lv->nbc[face]; ++j) {
            int64_t i = lv->bclist[face][j];
            double g[19];
            for (int k = 0; k < 19; ++k) {
                int m = tb ? k : INV[k];
                int64_t src = m == 0 ? i : pull_src(c, lv, 0, i, m);
                g[k] = src >= 0 ? lv->fcol[m * n + src] : lv->f[m * n + i];
            }
            if (face == 0) {
                double rho = (g[0] + g[3] + g[4] + g[5] + g[6] + g[15] + g[16] + g[17] + g[18] +
                              2.0 * (g[2] + g[8] + g[10] + g[12] + g[14])) / (1.0 - Ux);
                double ny = 0.5 * (g[3] + g[15] + g[17] - g[4] - g[16] - g[18]) - rho * Uy / 3.0;
                double nz = 0.5 * (g[5] + g[15] + g[18] - g[6] - g[16] - g[17]) - rho * Uz / 3.0;
                g[1] = g[2] + rho * Ux / 3.0;
                g[7] = g[8] + rho * (Ux + Uy) / 6.0 - ny;
                g[9] = g[10] + rho * (Ux - Uy) / 6.0 + ny;
                g[11] = g[12] + rho * (Ux + Uz) / 6.0 - nz;
                g[13] = g[14] + rho * (Ux - Uz) / 6.0 + nz;
            } else {
                int64_t nb = find_idx(lv, find_neighbor(c, lv->key[i], 0, -1, 0, 0));
                if (nb < 0) return -6;
                for (int t = 0; t < 5; ++t) {
                    int k = HH_IN_E[t];
                    int m = tb ? k : INV[k];
                    g[k] = lv->f[m * n + nb];
                }
            }
            for (int k = 0; k < 19; ++k) lv->f[(tb ? k : INV[k]) * n + i] = g[k];
        }
    }
    double feq[27], rho, u[3];
    const double tau0 = c->tau[0];
    for (int face = 0; face < 2; ++face)
        for (int64_t j = 0; j < lv->nbc[face]; ++j) {
            int64_t i = lv->bclist[face][j];
            double d[27];
            for (int k = 0; k < 19; ++k) d[k] = lv->f[k * n + i];
            macros_of(19, d, &rho, u);
            feq_bgk(19, rho, u, feq);
            for (int k = 0; k < 19; ++k) {
                double fk = d[k];
                lv->fcol[k * n + i] = fk - (fk - feq[k]) / tau0;
            }
        }
    return 0;
}

/* Interface time options of the device path (no reference counterpart; the
 * reference explodes in the first substep only, LBM_Simulator.cpp:47-51,
 * 122-125): 1 (MT_ITIME_HOLD) explodes in the second substep too from the
 * same parent values; 2 (MT_ITIME_EXTRAP) explodes the second substep from
 * the parent's values extrapolated to the half step, 1.5 fcol(t) - 0.5
 * fcol(t - 1), fcol(t - 1) being the sources' values at the parent's
 * previous step (the current values when the state was just set). */
int oc_set_interface_time(void *h, int mode)
{
    oc_case *c = (oc_case *)h;
    if (mode < 0 || mode > 2) return -1;
    c->itime = mode;
    c->prev_stale = 1;
    return 0;
}

/* Velocity of one face strategy (the input_v of
 * nonEquilibrumExtrapolation_<face>, NonEquilibrumExtrapolation.hpp:37-100)
 * and the face's boundary cells reset to f = fcol = feq(rho0, u) as
 * D3Q19_BC_Strategy::initial_Feq does (D3Q19_BC_Manager.hpp:157-167). */
int oc_set_face_velocity(void *h, int face, const double *u)
{
    oc_case *c = (oc_case *)h;
    if (face < 0 || face > 5) return -1;
    oc_level *lv = &c->lv[0];
    double feq[27];
    for (int a = 0; a < 3; ++a) c->face_u[face][a] = u[a];
    feq_bgk(c->q, c->rho0, u, feq);
    for (int g = 0; g < 9; ++g) {
        int b = FACE_SETS[face][g];
        if (b < 0) break;
        for (int64_t j = 0; j < lv->nbc[b]; ++j) {
            int64_t i = lv->bclist[b][j];
            for (int k = 0; k < c->q; ++k) {
                lv->f[k * lv->n + i] = feq[k];
                lv->fcol[k * lv->n + i] = feq[k];
            }
        }
    }
    return 0;
}

/* LBM_Manager::LBMkernel (LBM_Simulator.cpp:20-229) */
static int lbm_kernel(oc_case *c, int l)
{
    int rc;
    int L = c->L;
    for (int sub = 0; sub < 2; ++sub) {
        phase_macros(c, l);
        phase_collide(c, l);
        if (l == 0 && c->bc_mode == BC_ZOUHE_OUTFLOW)
            if ((rc = phase_bc_inout(c))) return rc;
        if (l < L)
            if ((rc = lbm_kernel(c, l + 1))) return rc;
        if ((sub == 0 || c->itime) && l > 0)
            if ((rc = phase_explosion(c, l, sub == 1 && c->itime == 2))) return rc;
        phase_stream(c, l);
        if (l == 0) {
            if (c->bc_mode == BC_NEQ)
                if ((rc = phase_bc_neq(c))) return rc;
            if (c->bc_mode == BC_ZOUHE_HH)
                if ((rc = phase_bc_hh(c))) return rc;
        } else if (l == L) {
            phase_ib(c);
        }
        if (l < L)
            if ((rc = phase_coalescence(c, l))) return rc;
        if (l == 0) break;
    }
    return 0;
}

/* LBM_Manager::fluidSimulate loop body (LBM_Simulator.cpp:11-17) without
 * diagnostics: one coarse step, then the all-level macroscopic update. */
int oc_step(void *h, int n_coarse)
{
    oc_case *c = (oc_case *)h;
    if (c->itime == 2 && c->prev_stale) {
        for (int l = 1; l <= c->L; ++l) save_sources(c, l);
        c->prev_stale = 0;
    }
    for (int s = 0; s < n_coarse; ++s) {
        int rc = lbm_kernel(c, 0);
        if (rc) return rc;
        for (int l = 0; l <= c->L; ++l) phase_macros(c, l);
    }
    return 0;
}

/* Neighbour table (level, cell, q) -> index or -1, pull convention */
int oc_neighbors(void *h, int level, int32_t *out)
{
    oc_case *c = (oc_case *)h;
    oc_level *lv = &c->lv[level];
    for (int64_t i = 0; i < lv->n; ++i)
        for (int k = 1; k < c->q; ++k) out[(k - 1) * lv->n + i] = (int32_t)pull_src(c, lv, level, i, k);
    return 0;
}

/* raw Morton neighbour keys for known-answer tests */
void oc_neighbor_keys(void *h, int level, const uint64_t *keys, int64_t n, uint64_t *out)
{
    oc_case *c = (oc_case *)h;
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < c->q; ++k) out[i * c->q + k] = find_neighbor(c, keys[i], level, EX[k], EY[k], EZ[k]);
}

/* single-cell collision kernel for known-answer tests */
void oc_collide_cell(int q, int collision, const double *f, double rho, const double *u, double tau, double *out)
{
    if (collision == COLL_LBGK) {
        double feq[27];
        feq_bgk(q, rho, u, feq);
        for (int k = 0; k < q; ++k) out[k] = f[k] - (f[k] - feq[k]) / tau;
    } else {
        cumulant_collide(f, rho, u, tau, out);
    }
}
