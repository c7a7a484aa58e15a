// Reference-style program over the drop-in header: the index sets go into
// the Lat_Manager singleton in bulk, LBM_Manager() is constructed without
// arguments from LBM_Manager::config(), and after fluidSimulate a loop shaped
// like LBM_Manager::infoPrint (LBM_Manager.cpp:914-981) reads
// user[l].velocity.at(code) and user[l].density.at(code) over every level's
// lat_f; then one population is changed through user[0].df.f[q].at(code)
// and one more coarse step is taken; then a checkpoint is saved and loaded
// back, and the steps after it must repeat bit for bit.
// usage: user_view_demo <sets.bin> <out.bin> <steps> <tau0> [tau1 ...]
// sets.bin uses the reference-harness input layout (oracle/oracle.py).
// out.bin: per level n, rho[n], ux[n], uy[n], uz[n] on lat_f (ascending key),
// max|v|; the changed key, direction and value; then per level the f [Q][n]
// of every stored cell after the extra step.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "mt_lbm.hpp"

template <class T> static T rd(FILE *f)
{
    T v;
    if (fread(&v, sizeof v, 1, f) != 1) throw std::runtime_error("short read");
    return v;
}

int main(int argc, char **argv)
{
    if (argc < 5) return 2;
    FILE *in = std::fopen(argv[1], "rb");
    if (!in) return 2;
    const int steps = std::atoi(argv[3]);
    mt_case_desc &d = mt::LBM_Manager::config();
    d.q = rd<int32_t>(in);
    d.max_level = rd<int32_t>(in);
    d.collision = rd<int32_t>(in);
    d.ib_method = rd<int32_t>(in);
    rd<int32_t>(in);  // steps recorded for the harness
    rd<int32_t>(in);  // warm-up steps
    rd<double>(in);   // viscosity (the relaxation times come from argv)
    for (int a = 0; a < 3; ++a) d.u_bc[a] = rd<double>(in);
    rd<double>(in);   // reference velocity
    d.bc_mode = MT_BC_NEQ;
    d.stream_convention = MT_PULL_REFERENCE;
    d.storage = MT_STORE_F64;
    d.rho0 = 1.0;
    d.extent0[0] = d.extent0[1] = d.extent0[2] = 1 << 10;
    for (int l = 0; l <= d.max_level; ++l) d.tau[l] = std::atof(argv[4 + l]);
    mt::Lat_Manager lat;
    for (int l = 0; l <= d.max_level; ++l)
        for (int s = 0; s < 6; ++s) {
            int64_t n = rd<int64_t>(in);
            std::vector<uint64_t> keys((size_t)n);
            for (auto &k : keys) k = rd<uint64_t>(in);
            std::vector<mt::Cell> cells((size_t)n, mt::Cell{s});
            mt::D_mapLat *sets[6] = {&lat.lat_f[l], &lat.lat_overlap_F2C[l], &lat.lat_overlap_C2F[l],
                                     &lat.ghost_overlap_C2F[l], &lat.ghost_overlap_F2C[l], &lat.lat_sf};
            sets[s]->insert_bulk(keys, cells);
        }
    for (int b = 0; b < 26; ++b) {
        int64_t n = rd<int64_t>(in);
        for (int64_t i = 0; i < n; ++i) lat.lat_bc[b].push_back(rd<uint64_t>(in));
    }
    int64_t nd = rd<int64_t>(in);
    for (int64_t i = 0; i < nd; ++i) {
        uint64_t k = rd<uint64_t>(in);
        std::vector<double> row(d.q - 1);
        for (auto &v : row) v = rd<double>(in);
        lat.dis.insert(std::make_pair(k, row));
    }
    std::fclose(in);
    try {
        mt::LBM_Manager mgr;
        if (mt::LBM_Manager::pointer_me != &mgr || mt::Lat_Manager::pointer_me != &lat) {
            std::fprintf(stderr, "pointer_me not set\n");
            return 1;
        }
        mgr.fluidSimulate(steps);
        FILE *out = std::fopen(argv[2], "wb");
        mt::LBM_Manager *m = mt::LBM_Manager::pointer_me;
        for (int l = 0; l <= d.max_level; ++l) {
            std::vector<double> rho, ux, uy, uz;
            double maxv = 0.0;
            for (auto i_lat : mt::Lat_Manager::pointer_me->lat_f.at(l)) {
                const mt::morton lat_code = i_lat.first;
                mt::D_uvw v = m->user[l].velocity.at(lat_code);
                const double vmag = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
                if (vmag > maxv) maxv = vmag;
                rho.push_back(m->user[l].density.at(lat_code));
                ux.push_back(v.x);
                uy.push_back(v.y);
                uz.push_back(v.z);
            }
            int64_t n = (int64_t)rho.size();
            std::fwrite(&n, 8, 1, out);
            for (auto *a : {&rho, &ux, &uy, &uz}) std::fwrite(a->data(), 8, a->size(), out);
            std::fwrite(&maxv, 8, 1, out);
        }
        // change one population of the first lat_f cell of level 0, then step
        const mt::morton code = lat.lat_f[0].begin()->first;
        const int q = 3;
        double &fq = m->user[0].df.f[q].at(code);
        fq += 1e-3;
        const double newv = m->user[0].df.f[q].at(code);
        const uint64_t ck = code.to_ullong();
        const int64_t qq = q;
        std::fwrite(&ck, 8, 1, out);
        std::fwrite(&qq, 8, 1, out);
        std::fwrite(&newv, 8, 1, out);
        mgr.fluidSimulate(1);
        for (int l = 0; l <= d.max_level; ++l) {
            std::vector<double> f, fcol;
            mgr.populations(l, f, fcol);
            int64_t n = (int64_t)f.size();
            std::fwrite(&n, 8, 1, out);
            std::fwrite(f.data(), 8, f.size(), out);
        }
        std::fclose(out);
        bool threw = false;
        try {
            m->user[0].df.f[q].at(uint64_t(0x7FFFFFFFFFFFFFFFull));
        } catch (const std::out_of_range &) {
            threw = true;
        }
        if (!threw) {
            std::fprintf(stderr, "missing key did not throw\n");
            return 1;
        }
        // checkpoint: save, two more steps; load it back, the same two
        // steps: the same populations, bit for bit
        const std::string ck_path = std::string(argv[2]) + ".ckpt";
        mgr.saveCheckpoint(ck_path);
        mgr.fluidSimulate(2);
        std::vector<std::vector<double>> fa(d.max_level + 1), fca(d.max_level + 1);
        for (int l = 0; l <= d.max_level; ++l) mgr.populations(l, fa[l], fca[l]);
        mgr.loadCheckpoint(ck_path);
        mgr.fluidSimulate(2);
        for (int l = 0; l <= d.max_level; ++l) {
            std::vector<double> f, fcol;
            mgr.populations(l, f, fcol);
            if (f != fa[l] || fcol != fca[l]) {
                std::fprintf(stderr, "resumed level %d differs\n", l);
                return 1;
            }
        }
        const int64_t st = mgr.coarseSteps();
        if (st != steps + 1 + 2) {
            std::fprintf(stderr, "step count %lld after resume\n", (long long)st);
            return 1;
        }
        std::remove(ck_path.c_str());
    } catch (const std::exception &e) {
        std::fprintf(stderr, "user_view_demo: %s\n", e.what());
        return 1;
    }
    return 0;
}
