/*
 * Case configuration header for the reference harness.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference reads its whole configuration
 * from compile-time constants in header/Constants.h (one namespace per
 * case, selected with `using namespace sphere;`, Constants.h:37-467).  The
 * harness compiles the reference's own LBM translation units against this
 * file instead, so the constants below keep the reference's names (the
 * translation units refer to them, some as `sphere::C_IB_use_FH`) while
 * the lattice and the level count come from -D flags chosen per harness
 * binary (HC_Q = 19 or 27, HC_L = maximum refinement level).  Viscosity and
 * velocities are single-definition variables that the harness sets from
 * its input file before it constructs LBM_Manager.
 *
 * Grid spacing and time step are 1 (lattice units at level 0), so the
 * conversion factor of velocity is 1 and tau_l = 3 nu 2^l + 1/2.
 */
#pragma once

#include "General.h"

#define C_DEBUG 0
#define C_CHECK_MORTON_BOUNDARY 0
#define C_SPEED_UP 0
#define C_MAP_TYPE 1
#define USE_HASHMAP
#define C_SEARCH_METHOD 1
#define C_FSI_INTERFACE 0
#define C_SOLID_BOUNDARY 1

#ifndef HC_Q
#define HC_Q 19
#endif
#ifndef HC_L
#define HC_L 1
#endif

namespace sphere
{
    const std::string F_model_path = "unused.stl";
    const std::string OUTPUT_NAME = "harness";

    #define C_DIMS 3
    #define C_Q HC_Q

    constexpr D_real C_xb = 1;
    constexpr D_real C_yb = 1;
    constexpr D_real C_zb = 1;
    constexpr D_real xb_domain = C_xb;
    constexpr D_real yb_domain = C_yb;
    constexpr D_real zb_domain = C_zb;
    constexpr D_real C_domain[6] = {0, 0, 0, C_xb, C_yb, C_zb};
    constexpr D_real C_solid_origin[3] = {0, 0, 0};

    constexpr D_real C_dx = 1.0;
    constexpr int C_x0b_offset = 0;
    constexpr int C_y0b_offset = 0;
    constexpr int C_z0b_offset = 0;
    constexpr uint C_max_level = HC_L;
    constexpr bool C_IB_use_FH = true;
    constexpr uint C_overlap = 1;
    constexpr uint C_extend_inner = 2;
    constexpr uint C_extend_inner_x0 = 2;
    constexpr uint C_extend_inner_x1 = 2;
    constexpr uint C_extend_inner_y0 = 2;
    constexpr uint C_extend_inner_y1 = 2;
    constexpr uint C_extend_inner_z0 = 2;
    constexpr uint C_extend_inner_z1 = 2;
    constexpr uint C_extend = 4;
    constexpr uint C_extend_outer_x0 = 2;
    constexpr uint C_extend_outer_x1 = 2;
    constexpr uint C_extend_outer_y0 = 2;
    constexpr uint C_extend_outer_y1 = 2;
    constexpr uint C_extend_outer_z0 = 2;
    constexpr uint C_extend_outer_z1 = 2;
    constexpr uint C_extend_ghost = 0;

    constexpr uint U_iters = 1;
    constexpr uint U_outputIters = 1000000;

    static D_real U_dt = 1.0;

    inline D_real U_u0 = 0.05;
    inline D_real U_v0 = 0.;
    inline D_real U_w0 = 0.;
    constexpr D_real U_rho0 = 1.;
    inline D_real U_kineViscosity = 0.02;
    inline D_real U_dynaViscosity = 0.02;

    inline D_real R_velocity = 0.05;
    constexpr D_real R_length = 1.;
    inline D_real R_Re = 1.;
}

using namespace sphere;

constexpr D_real MAX_MACH = 0.09;
constexpr D_real MIN_TAU = 0.500001;

/* Lattice velocity sets in the reference's direction order. */
#if (C_Q == 19)
constexpr int ex[C_Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
constexpr int ey[C_Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
constexpr int ez[C_Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
constexpr unsigned int e_inv[C_Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
#elif (C_Q == 27)
constexpr int ex[C_Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0,
                         1, -1, 1, -1, -1, 1, -1, 1};
constexpr int ey[C_Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1,
                         1, -1, -1, 1, -1, 1, 1, -1};
constexpr int ez[C_Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1,
                         1, -1, 1, -1, 1, -1, 1, -1};
constexpr unsigned int e_inv[C_Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17,
                                     20, 19, 22, 21, 24, 23, 26, 25};
#endif
