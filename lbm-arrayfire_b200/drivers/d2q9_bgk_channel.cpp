// d2q9_bgk_channel.cpp — headless version of the reference's D2Q9 BGK channel with a cylinder
// (cpp/d2q9_bgk_channel_packed.cpp, the copy of cpp/d2q9_bgk_channel.cpp with the correct ey) on
// liblbm_b200.  The loop body (stream, macros, inlet/solid/end-column overwrites, equilibrium, BGK,
// bounce-back; :54-74) is one lbm_step call per reporting interval.  Same geometry and parameters as
// the reference (:10-19: 700 x 300, cylinder at (nx/5 + 1, ny/2 + ny/30) of radius ny/10 + 1, Re 220,
// u_max 0.1, nu = u_max 2 r / Re) and the same start state (:44-48: DENSITY = rho0, UX = u_max,
// UY = 0, with UX(ON) = DENSITY(ON) = 0).  The reference loops until its window closes; this one runs
// a given number of iterations and prints the reference's console report (the C++ lid driver's
// format, MLUPS formula corrected).  Options:
//   --config      config-mode boundaries: equilibrium inlet and zero-gradient outlet instead of the
//                 reference's periodic channel with forced end columns
//   --zouhe       Zou-He velocity inlet and pressure outlet (rho = 1) instead
//   --csv PATH    "Iterations,MLUPS" every 100 iterations
//   --dump PATH   final DENSITY, UX, UY as raw float64 [N | N | N], column-major
//
//   d2q9_bgk_channel [nx ny iterations] [--re R] [--u U] [--storage f32|f16s|bf16s] [--config|--zouhe]
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "lbm.h"

static int fail(const char* what) {
    std::fprintf(stderr, "%s: %s\n", what, lbm_last_error());
    return 1;
}

int main(int argc, char** argv) {
    long long nx = 700, ny = 300, maxiter = 1000;
    double re = 220.0, u_max = 0.1;
    int storage = LBM_F32, config_mode = 0;
    std::string csv, dump;
    int pos = 0;
    for (int a = 1; a < argc; ++a) {
        const std::string s = argv[a];
        if (s == "--re" && a + 1 < argc) re = std::atof(argv[++a]);
        else if (s == "--u" && a + 1 < argc) u_max = std::atof(argv[++a]);
        else if (s == "--csv" && a + 1 < argc) csv = argv[++a];
        else if (s == "--dump" && a + 1 < argc) dump = argv[++a];
        else if (s == "--config") config_mode = 1;
        else if (s == "--zouhe") config_mode = 2;
        else if (s == "--storage" && a + 1 < argc) {
            const std::string v = argv[++a];
            storage = v == "f16s" ? LBM_F16S : v == "bf16s" ? LBM_BF16S : LBM_F32;
        } else if (pos == 0) nx = std::atoll(s.c_str()), ++pos;
        else if (pos == 1) ny = std::atoll(s.c_str()), ++pos;
        else if (pos == 2) maxiter = std::atoll(s.c_str()), ++pos;
    }
    const long long total_nodes = nx * ny;
    const long long ox = nx / 5 + 1, oy = ny / 2 + ny / 30, r = ny / 10 + 1;  // integer, as at :13-15
    const double nu = u_max * 2 * r / re;
    const double tau = 3 * nu + 0.5;
    const double omega = 1.0 / tau;
    std::printf("LBM D2Q9 channel simulation\n");
    std::printf("Lattice: %lld x %lld, cylinder at (%lld, %lld), radius %lld\n", nx, ny, ox, oy, r);
    std::printf("Inlet velocity u_max: %f\n", u_max);
    std::printf("Reynolds number: %f\n", re);
    std::printf("Lattice viscosity: %f\n", nu);
    std::printf("Relaxation time: %f\n", tau);
    std::printf("Relaxation parameter: %f\n", omega);

    lbm_desc d;
    lbm_desc_init(&d, LBM_D2Q9, LBM_BGK, storage, nx, ny, 1);
    d.omega = omega;
    std::vector<uint8_t> mask((size_t)total_nodes);
    if (lbm_setup_channel2d(&d, mask.data(), u_max, (double)ox, (double)oy, (double)r, config_mode) != LBM_OK)
        return fail("lbm_setup_channel2d");
    lbm_ctx* ctx = nullptr;
    if (lbm_create(&d, &ctx) != LBM_OK) return fail("lbm_create");
    // DENSITY = rho0, UX = u_max, UY = 0; UX(ON) = 0, DENSITY(ON) = 0 (:44-48)
    std::vector<double> rho0((size_t)total_nodes), u0((size_t)(2 * total_nodes), 0.0);
    for (long long k = 0; k < total_nodes; ++k) {
        const bool solid = (d.classes[mask[k]].flags & LBM_CELL_BOUNCE) != 0;
        rho0[k] = solid ? 0.0 : 1.0;
        u0[k] = solid ? 0.0 : u_max;
    }
    if (lbm_init_equilibrium(ctx, rho0.data(), u0.data()) != LBM_OK) return fail("lbm_init_equilibrium");

    FILE* fcsv = csv.empty() ? nullptr : std::fopen(csv.c_str(), "w");
    if (fcsv) std::fprintf(fcsv, "Iterations,MLUPS\n");
    const auto t0 = std::chrono::steady_clock::now();
    long long iter = 0;
    while (iter < maxiter) {
        const long long n = std::min<long long>(100 - iter % 100, maxiter - iter);
        if (lbm_step(ctx, n) != LBM_OK) return fail("lbm_step");
        iter += n;
        if (iter % 100 == 0) {
            if (lbm_sync(ctx) != LBM_OK) return fail("lbm_sync");
            const double time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            const double mlups = total_nodes * (double)iter * 1e-6 / time;
            std::printf("%lld iterations completed, %fs elapsed (%f MLUPS).\n", iter, time, mlups);
            if (fcsv) std::fprintf(fcsv, "%lld,%f\n", iter, mlups);
        }
    }
    if (lbm_sync(ctx) != LBM_OK) return fail("lbm_sync");
    const double end = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("Iterations: %lld\n", iter);
    std::printf("Time: %fs\n", end);
    std::printf("MLUPS: %f\n", total_nodes * (double)iter * 1e-6 / end);
    if (fcsv) std::fclose(fcsv);

    if (!dump.empty()) {
        std::vector<double> rho((size_t)total_nodes), u((size_t)(2 * total_nodes));
        if (lbm_get_macros(ctx, rho.data(), u.data(), LBM_DTYPE_F64, LBM_HOST) != LBM_OK) return fail("lbm_get_macros");
        FILE* f = std::fopen(dump.c_str(), "wb");
        if (!f) return fail("dump file");
        std::fwrite(rho.data(), sizeof(double), rho.size(), f);
        std::fwrite(u.data(), sizeof(double), u.size(), f);
        std::fclose(f);
    }
    lbm_destroy(ctx);
    return 0;
}
