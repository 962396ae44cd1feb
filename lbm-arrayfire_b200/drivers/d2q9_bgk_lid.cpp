// d2q9_bgk_lid.cpp — headless version of the reference's D2Q9 BGK lid-driven cavity driver
// (cpp/d2q9_bgk_lid.cpp) on liblbm_b200: the loop body (stream, macros, lid/solid overwrites,
// equilibrium, BGK, bounce-back; :123-155) is one lbm_step call per reporting interval.  Same
// parameters and console report as the reference (:36-56, :172-188), with the MLUPS formula
// corrected (the reference multiplies by 10e-6 instead of 1e-6), no window, and optional outputs:
//   --csv PATH    "Iterations,MLUPS" every 100 iterations (the Rust drivers' benchmark file)
//   --dump PATH   final DENSITY, UX, UY as raw float64 [N | N | N], column-major
//
//   d2q9_bgk_lid [nx ny iterations] [--re R] [--u U] [--storage f32|f16s|bf16s] [--rust-nu]
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lbm.h"

static int fail(const char* what) {
    std::fprintf(stderr, "%s: %s\n", what, lbm_last_error());
    return 1;
}

int main(int argc, char** argv) {
    long long nx = 256, ny = 256, maxiter = 1000;
    double re = 200.0, ux_lid = 0.05;
    int storage = LBM_F32, rule = 0;
    std::string csv, dump;
    int pos = 0;
    for (int a = 1; a < argc; ++a) {
        const std::string s = argv[a];
        if (s == "--re" && a + 1 < argc) re = std::atof(argv[++a]);
        else if (s == "--u" && a + 1 < argc) ux_lid = std::atof(argv[++a]);
        else if (s == "--csv" && a + 1 < argc) csv = argv[++a];
        else if (s == "--dump" && a + 1 < argc) dump = argv[++a];
        else if (s == "--rust-nu") rule = 1;
        else if (s == "--storage" && a + 1 < argc) {
            const std::string v = argv[++a];
            storage = v == "f16s" ? LBM_F16S : v == "bf16s" ? LBM_BF16S : LBM_F32;
        } else if (pos == 0) nx = std::atoll(s.c_str()), ++pos;
        else if (pos == 1) ny = std::atoll(s.c_str()), ++pos;
        else if (pos == 2) maxiter = std::atoll(s.c_str()), ++pos;
    }
    const long long total_nodes = nx * ny;
    const double nu = ux_lid * (rule ? 2.0 : 1.0) * nx / re;
    const double tau = 3 * nu + 0.5;
    const double omega = lbm_omega_from_re(ux_lid, (double)nx, re, rule);
    std::printf("LBM D2Q9 simulation\n");
    std::printf("Horizontal lid velocity ux_lid: %f\n", ux_lid);
    std::printf("Vertical lid velocity uy_lid: %f\n", 0.0);
    std::printf("Reynolds number: %f\n", re);
    std::printf("Lattice viscosity: %f\n", nu);
    std::printf("Relaxation time: %f\n", tau);
    std::printf("Relaxation parameter: %f\n", omega);

    lbm_desc d;
    lbm_desc_init(&d, LBM_D2Q9, LBM_BGK, storage, nx, ny, 1);
    d.omega = omega;
    std::vector<uint8_t> mask((size_t)total_nodes);
    if (lbm_setup_cavity2d(&d, mask.data(), ux_lid) != LBM_OK) return fail("lbm_setup_cavity2d");
    lbm_ctx* ctx = nullptr;
    if (lbm_create(&d, &ctx) != LBM_OK) return fail("lbm_create");
    // DENSITY = 1, UX = UY = 0 everywhere, solids included (:100-107)
    if (lbm_init_equilibrium(ctx, nullptr, nullptr) != LBM_OK) return fail("lbm_init_equilibrium");
    if (lbm_sync(ctx) != LBM_OK) return fail("lbm_sync");

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
