/*
 * harness.cpp -- drives the reference's own LBM translation units
 * (LBM_Manager.cpp, LBM_Simulator.cpp, lbm_kernel/*, BC/*,
 * ComplexBoundary_Manager.cpp, Morton_Assist.cpp) on index sets supplied in
 * a binary file, and dumps the populations it produces.
 *
 * TEST INFRASTRUCTURE ONLY: it generates the golden vectors that pin the
 * oracle and times the reference CPU path.  The reference mesher cannot
 * produce box-refined meshes (Grid_Manager.cpp:99-102 leaves intermediate
 * levels empty), so the harness fills Lat_Manager's public sets directly and
 * sets dx[l] on every level (the reference only sets the finest one,
 * Lat_Voxelize.cpp:422), then runs LBM_Manager::LBMkernel(0) followed by the
 * all-level macroscopic update, i.e. the body of LBM_Manager::fluidSimulate
 * (LBM_Simulator.cpp:8-18) without the diagnostics print and Tecplot output.
 *
 * usage: harness step  <in.bin> <out.bin>
 *        harness pstep <in.bin> <out.bin>      (step with periodic axes)
 *        harness trace <in.bin> <out.bin>      (state dumps after chosen steps)
 *        harness tecplot <in.bin> <out.bin>    (the reference's flow file after the steps)
 *        harness dis <in.bin> <out.bin>        (wall distances by compute_distance)
 *        harness morton <in.bin> <out.bin>     (neighbour-key known answers)
 *
 * Built with -DHC_PERIODIC the harness includes a generated copy of
 * Morton_Assist.h whose find_neighbor wraps the level-0 box on the axes the
 * trace input marks periodic (the reference has no periodic path that
 * builds, BC/Periodic.cpp needs the ghost layers that BC_NO_GHOST removes);
 * with no axis marked it is the reference's arithmetic unchanged.
 */
#include <sys/stat.h>

#include <algorithm>
#include <array>
#include <bitset>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <vector>

/* the harness reaches LBM_Manager's private stepping entry point and state */
#define private public
#define protected public
#include "General.h"
#include "Constants.h"
#include "Morton_Assist.h"
#include "Lat_Manager.hpp"
#include "LBM_Manager.hpp"
#include "IO_Manager.h"
#include "lbm_kernel/Collision_Model_Factory.hpp"
#include "lbm_kernel/Stream_Manager.hpp"
#include "ComplexBoundary_Manager.hpp"
#include "BC/D3Q19_BC_Manager.hpp"
#undef private
#undef protected
#include "Grid_Manager.h"
#include "Solid_Manager.h"
#include "Shape.h"

/* static members whose definitions live in translation units the harness
 * does not build (Grid_Manager.cpp, Lat_Manager.cpp, Obj_Manager.cpp ...) */
Morton_Assist *Morton_Assist::pointer_me;
std::array<D_morton, C_max_level + 1> Morton_Assist::ref_one;
std::array<std::array<D_morton, 2>, C_max_level + 1> Morton_Assist::xmorton_ref;
std::array<std::array<D_morton, 2>, C_max_level + 1> Morton_Assist::ymorton_ref;
std::array<std::array<D_morton, 2>, C_max_level + 1> Morton_Assist::zmorton_ref;
std::array<D_morton, C_max_level + 1> Morton_Assist::morton_xyz;
std::array<D_morton, C_max_level + 1> Morton_Assist::morton_xyz_flip;
D_morton Morton_Assist::mortonx_min, Morton_Assist::mortonx_max;
D_morton Morton_Assist::mortony_min, Morton_Assist::mortony_max;
D_morton Morton_Assist::mortonz_min, Morton_Assist::mortonz_max;
Lat_Manager *Lat_Manager::pointer_me;
LBM_Manager *LBM_Manager::pointer_me;
IO_Manager *IO_Manager::pointer_me;
/* tecplot.cpp's mesh writers name these; the flow writer used here does not */
Grid_Manager *Grid_Manager::pointer_me;
Solid_Manager *Solid_Manager::pointer_me;
std::ofstream *Log_function::logfile;
void IO_Manager::writeFlow(const D_int) {}

namespace {

struct Reader {
    FILE *fp;
    template <class T> T get()
    {
        T v;
        if (fread(&v, sizeof(T), 1, fp) != 1) throw std::runtime_error("short input");
        return v;
    }
    template <class T> std::vector<T> vec(int64_t n)
    {
        std::vector<T> v((size_t)n);
        if (n && fread(v.data(), sizeof(T), (size_t)n, fp) != (size_t)n) throw std::runtime_error("short input");
        return v;
    }
};

D_morton K(uint64_t k) { return D_morton(k); }

void setup_morton(Morton_Assist &ma)
{
    Morton_Assist::pointer_me = &ma;
    ma.morton_initial();
    for (unsigned l = 0; l <= C_max_level; ++l) Morton_Assist::compute_ref(l);
}

int run_morton(Reader &in, FILE *out)
{
    Morton_Assist ma;
    setup_morton(ma);
    int64_t n = in.get<int64_t>();
    auto lev = in.vec<int32_t>(n);
    auto keys = in.vec<uint64_t>(n);
    for (int64_t i = 0; i < n; ++i)
        for (int q = 0; q < C_Q; ++q) {
            uint64_t r = Morton_Assist::find_neighbor(K(keys[i]), (uint)lev[i], ex[q], ey[q], ez[q]).to_ullong();
            fwrite(&r, 8, 1, out);
        }
    return 0;
}

struct Loaded {
    LBM_Manager *mgr = nullptr;
    int32_t L = 0, nsteps = 0, nwarm = 0;
};

/* reads the case (index sets, parameters, optional initial populations) and
 * constructs the reference's LBM_Manager on it */
int load_case(Reader &in, Loaded &c)
{
    int32_t q = in.get<int32_t>(), L = in.get<int32_t>();
    if (q != C_Q || L != (int32_t)C_max_level) {
        fprintf(stderr, "harness built for Q=%d L=%d, input has Q=%d L=%d\n", C_Q, (int)C_max_level, q, L);
        return 2;
    }
    int32_t collision = in.get<int32_t>(), ib_fh = in.get<int32_t>(), nsteps = in.get<int32_t>();
    int32_t nwarm = in.get<int32_t>();
    sphere::U_kineViscosity = in.get<double>();
    sphere::U_u0 = in.get<double>();
    sphere::U_v0 = in.get<double>();
    sphere::U_w0 = in.get<double>();
    sphere::R_velocity = in.get<double>();
    sphere::U_dynaViscosity = sphere::U_kineViscosity * U_rho0;
    sphere::R_Re = sphere::R_velocity * R_length / sphere::U_kineViscosity;

    Lat_Manager *lm = new Lat_Manager();
    Lat_Manager::pointer_me = lm;
    std::array<D_mapLat, C_max_level + 1> *maps[5] = {&lm->lat_f, &lm->lat_overlap_F2C, &lm->lat_overlap_C2F,
                                                     &lm->ghost_overlap_C2F, &lm->ghost_overlap_F2C};
    const int flags[5] = {FLUID, OVERLAP_F2C, OVERLAP_C2F, OVERLAP_GHOST, OVERLAP_GHOST};
    for (int l = 0; l <= L; ++l) {
        for (int s = 0; s < 6; ++s) {
            int64_t n = in.get<int64_t>();
            auto keys = in.vec<uint64_t>(n);
            for (auto k : keys) {
                if (s < 5)
                    (*maps[s])[l].insert(std::make_pair(K(k), Cell(flags[s])));
                else
                    lm->lat_sf.insert(std::make_pair(K(k), Cell(SOLID)));
            }
        }
        lm->dx[l] = C_dx / (double)two_power_n(l);
    }
    for (int b = 0; b < 26; ++b) {
        int64_t n = in.get<int64_t>();
        auto keys = in.vec<uint64_t>(n);
        for (auto k : keys) lm->lat_bc[b].insert(K(k));
    }
    {
        int64_t n = in.get<int64_t>();
        for (int64_t i = 0; i < n; ++i) {
            uint64_t k = in.get<uint64_t>();
            auto row = in.vec<double>(C_Q - 1);
            std::array<D_real, C_Q - 1> a;
            for (int j = 0; j < C_Q - 1; ++j) a[j] = row[j];
            lm->dis.insert(std::make_pair(K(k), a));
        }
    }

    LBM_Manager *mgr = new LBM_Manager();
    if (collision == 1) mgr->collideModel = Collision_Model_Factory::createCollisionModel("Cumulant");
    if (!ib_fh) mgr->solidBCModel = new SinglePointInterpolation(mgr->user, IB_Method::DISTANCE_WEIGHTED);
    mgr->initialBC();

    int32_t init_mode = in.get<int32_t>();
    if (init_mode == 1) {
        for (int l = 0; l <= L; ++l) {
            int64_t n = in.get<int64_t>();
            for (int64_t i = 0; i < n; ++i) {
                uint64_t k = in.get<uint64_t>();
                auto f = in.vec<double>(C_Q);
                for (int j = 0; j < C_Q; ++j) {
                    mgr->user[l].df.f[j].at(K(k)) = f[j];
                    mgr->user[l].df.fcol[j].at(K(k)) = f[j];
                }
            }
        }
    }
    c.mgr = mgr;
    c.L = L;
    c.nsteps = nsteps;
    c.nwarm = nwarm;
    return 0;
}

/* one coarse step as LBM_Manager::fluidSimulate takes it (LBM_Simulator.cpp:8-18),
 * then the step's IB force sum is appended and the accumulator cleared */
void coarse_step(LBM_Manager *mgr, std::vector<double> &force)
{
    mgr->LBMkernel(0);
    mgr->calculateMacros();
    force.push_back(mgr->m_ibFx_sum);
    force.push_back(mgr->m_ibFy_sum);
    force.push_back(mgr->m_ibFz_sum);
    force.push_back((double)mgr->m_ibForce_count);
    mgr->m_ibFx_sum = mgr->m_ibFy_sum = mgr->m_ibFz_sum = 0.0;
    mgr->m_ibForce_count = 0;
}

/* every stored cell of every level, ascending key: f[Q], fcol[Q], rho, u */
void write_levels(LBM_Manager *mgr, int L, FILE *out)
{
    for (int l = 0; l <= L; ++l) {
        std::vector<uint64_t> keys;
        for (auto &kv : mgr->user[l].df.f[0]) keys.push_back(kv.first.to_ullong());
        std::sort(keys.begin(), keys.end());
        int64_t n = (int64_t)keys.size();
        fwrite(&n, 8, 1, out);
        for (auto k : keys) {
            fwrite(&k, 8, 1, out);
            double rec[2 * C_Q + 4];
            for (int j = 0; j < C_Q; ++j) {
                rec[j] = mgr->user[l].df.f[j].at(K(k));
                rec[C_Q + j] = mgr->user[l].df.fcol[j].at(K(k));
            }
            auto d = mgr->user[l].density.find(K(k));
            auto v = mgr->user[l].velocity.find(K(k));
            rec[2 * C_Q] = d == mgr->user[l].density.end() ? NAN : d->second;
            rec[2 * C_Q + 1] = v == mgr->user[l].velocity.end() ? NAN : v->second.x;
            rec[2 * C_Q + 2] = v == mgr->user[l].velocity.end() ? NAN : v->second.y;
            rec[2 * C_Q + 3] = v == mgr->user[l].velocity.end() ? NAN : v->second.z;
            fwrite(rec, 8, 2 * C_Q + 4, out);
        }
    }
}

void write_tail(LBM_Manager *mgr, const std::vector<double> &force, FILE *out)
{
    int64_t nf = (int64_t)force.size();
    fwrite(&nf, 8, 1, out);
    fwrite(force.data(), 8, force.size(), out);
    double tau[C_max_level + 1];
    for (unsigned l = 0; l <= C_max_level; ++l) tau[l] = mgr->tau[l];
    fwrite(tau, 8, C_max_level + 1, out);
}

/* reads int32 periodic[3], int32 extent0[3] and turns the find_neighbor
 * wrap on (harness built with HC_PERIODIC) */
int read_periodic(Reader &in)
{
    int32_t per[3], ext[3];
    for (auto &p : per) p = in.get<int32_t>();
    for (auto &e : ext) e = in.get<int32_t>();
#ifdef HC_PERIODIC
    for (int a = 0; a < 3; ++a) {
        hc_periodic[a] = per[a];
        hc_extent0[a] = ext[a];
    }
#else
    if (per[0] || per[1] || per[2]) {
        fprintf(stderr, "periodic axes need the harness built with HC_PERIODIC\n");
        return 2;
    }
#endif
    return 0;
}

/* step (pstep: followed by the periodic section of read_periodic) */
int run_step(Reader &in, FILE *out, bool periodic = false)
{
    Morton_Assist ma;
    setup_morton(ma);
    Loaded c;
    if (int rc = load_case(in, c)) return rc;
    if (periodic)
        if (int rc = read_periodic(in)) return rc;
    LBM_Manager *mgr = c.mgr;
    std::vector<double> force;
    for (int s = 0; s < c.nwarm; ++s) {
        mgr->LBMkernel(0);
        mgr->calculateMacros();
    }
    mgr->m_ibFx_sum = mgr->m_ibFy_sum = mgr->m_ibFz_sum = 0.0;
    mgr->m_ibForce_count = 0;
    auto t0 = std::chrono::steady_clock::now();
    for (int s = 0; s < c.nsteps; ++s) coarse_step(mgr, force);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    fwrite(&secs, 8, 1, out);
    write_levels(mgr, c.L, out);
    write_tail(mgr, force, out);
    return 0;
}

/* dis: wall distances of chosen finest-level cells by the reference's own
 * Lat_Manager::compute_distance (Lat_Voxelize.cpp:1252-1285, through
 * Shape::intersect_line_with_triangle, Shape.cpp:809-843) over every given
 * triangle, the call Lat_Voxelize.cpp:848 makes for each triangle near an
 * immersed-boundary cell.  Input: int64 ntri, ntri x 9 doubles (coarse-cell
 * units), int64 ncell, per cell uint64 key + 3 doubles (its centre).
 * Output: per cell Q - 1 doubles, -1 where no link crosses. */
int run_dis(Reader &in, FILE *out)
{
    Morton_Assist ma;
    setup_morton(ma);
    Lat_Manager *lm = new Lat_Manager();
    Lat_Manager::pointer_me = lm;
    for (unsigned l = 0; l <= C_max_level; ++l) lm->dx[l] = C_dx / (double)two_power_n(l);
    const int64_t nt = in.get<int64_t>();
    std::vector<Solid_Face> tris((size_t)nt);
    for (auto &t : tris) {
        auto v = in.vec<double>(9);
        t.vertex1.x = v[0]; t.vertex1.y = v[1]; t.vertex1.z = v[2];
        t.vertex2.x = v[3]; t.vertex2.y = v[4]; t.vertex2.z = v[5];
        t.vertex3.x = v[6]; t.vertex3.y = v[7]; t.vertex3.z = v[8];
    }
    const int64_t nc = in.get<int64_t>();
    for (int64_t i = 0; i < nc; ++i) {
        const uint64_t k = in.get<uint64_t>();
        auto c = in.vec<double>(3);
        for (const auto &t : tris) lm->compute_distance(t, K(k), D_vec(c[0], c[1], c[2]));
        double row[C_Q - 1];
        auto it = lm->dis.find(K(k));
        for (int j = 0; j < C_Q - 1; ++j) row[j] = it == lm->dis.end() ? -1.0 : it->second[j];
        fwrite(row, 8, C_Q - 1, out);
    }
    return 0;
}

/* tecplot: the step input followed by int32 iter; after the steps the
 * reference's IO_TECPLOTH::write(iter) (tecplot.cpp:16-176) writes
 * output/sphereFlow_<iter * CF_T[0]>.dat under the working directory. */
int run_tecplot(Reader &in, FILE *out)
{
    Morton_Assist ma;
    setup_morton(ma);
    Loaded c;
    if (int rc = load_case(in, c)) return rc;
    const int32_t iter = in.get<int32_t>();
    std::vector<double> force;
    for (int s = 0; s < c.nsteps; ++s) coarse_step(c.mgr, force);
    mkdir(C_OUTPUT_DIR, 0777);
    IO_TECPLOTH tp;
    tp.write(iter);
    const int32_t done = 1;
    fwrite(&done, 4, 1, out);
    return 0;
}

/* trace: the step input followed by int32 ndump, int32 dump_after[ndump]
 * (ascending coarse-step counts), int32 periodic[3], int32 extent0[3]
 * (level-0 box).  Output: seconds, then the levels after each listed step,
 * then the per-step force series and tau. */
int run_trace(Reader &in, FILE *out)
{
    Morton_Assist ma;
    setup_morton(ma);
    Loaded c;
    if (int rc = load_case(in, c)) return rc;
    int32_t ndump = in.get<int32_t>();
    auto dumps = in.vec<int32_t>(ndump);
    if (int rc = read_periodic(in)) return rc;
    LBM_Manager *mgr = c.mgr;
    std::vector<double> force;
    double secs = 0;
    int32_t done = 0;
    for (int32_t d = 0; d < ndump; ++d) {
        auto t0 = std::chrono::steady_clock::now();
        for (; done < dumps[d]; ++done) coarse_step(mgr, force);
        secs += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        write_levels(mgr, c.L, out);
        fflush(out);
    }
    fwrite(&secs, 8, 1, out);
    write_tail(mgr, force, out);
    return 0;
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc != 4) {
        fprintf(stderr, "usage: %s step|pstep|trace|tecplot|dis|morton <in.bin> <out.bin>\n", argv[0]);
        return 2;
    }
    std::ofstream devnull("/dev/null");
    Log_function::logfile = &devnull;
    if (!freopen("/dev/null", "w", stdout)) return 3;
    FILE *fin = fopen(argv[2], "rb");
    FILE *fout = fopen(argv[3], "wb");
    if (!fin || !fout) return 3;
    Reader rd{fin};
    int rc;
    try {
        const std::string mode = argv[1];
        rc = mode == "morton"    ? run_morton(rd, fout)
             : mode == "trace"   ? run_trace(rd, fout)
             : mode == "tecplot" ? run_tecplot(rd, fout)
             : mode == "dis"     ? run_dis(rd, fout)
             : run_step(rd, fout, mode == "pstep");
    } catch (const std::exception &e) {
        fprintf(stderr, "harness: %s\n", e.what());
        rc = 4;
    }
    fclose(fout);
    fclose(fin);
    return rc;
}
