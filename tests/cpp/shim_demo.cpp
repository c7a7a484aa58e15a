// Drop-in demo: fill Lat_Manager's sets, build LBM_Manager, run
// fluidSimulate and dump the populations, through include/mt_lbm.hpp.
// usage: shim_demo <sets.bin> <out.bin> <steps> <tau0> [tau1 ...]
// sets.bin uses the reference-harness input layout (oracle/oracle.py).
#include <cstdio>
#include <cstdlib>
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
    mt_case_desc d{};
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
    for (int l = 0; l <= d.max_level; ++l) d.tau[l] = std::atof(argv[4 + l]);
    mt::Lat_Manager lat;
    for (int l = 0; l <= d.max_level; ++l)
        for (int s = 0; s < 6; ++s) {
            int64_t n = rd<int64_t>(in);
            for (int64_t i = 0; i < n; ++i) {
                uint64_t k = rd<uint64_t>(in);
                mt::D_mapLat *sets[5] = {&lat.lat_f[l], &lat.lat_overlap_F2C[l], &lat.lat_overlap_C2F[l],
                                         &lat.ghost_overlap_C2F[l], &lat.ghost_overlap_F2C[l]};
                if (s < 5)
                    sets[s]->insert(std::make_pair(k, mt::Cell{s}));
                else
                    lat.lat_sf.insert(std::make_pair(k, mt::Cell{s}));
            }
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
    // extents are only read for periodic axes; this demo uses the reference's boundary shell
    d.extent0[0] = d.extent0[1] = d.extent0[2] = 1 << 10;
    try {
        mt::Context ctx(0);
        mt::LBM_Manager mgr(ctx, lat, d);
        mgr.fluidSimulate(steps);
        FILE *out = std::fopen(argv[2], "wb");
        for (int l = 0; l <= d.max_level; ++l) {
            std::vector<double> f, fcol;
            mgr.populations(l, f, fcol);
            int64_t n = (int64_t)f.size();
            std::fwrite(&n, 8, 1, out);
            std::fwrite(f.data(), 8, f.size(), out);
        }
        auto fo = mgr.force();
        std::fwrite(fo.data(), 8, 4, out);
        std::fclose(out);
        std::printf("%s steps=%d\n", mgr.collideModel->print_Model_Name().c_str(), steps);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "shim_demo: %s\n", e.what());
        return 1;
    }
    return 0;
}
