// d3q27_bgk_lid.cpp — headless version of the reference's D3Q27 BGK lid-driven cavity driver
// (cpp/d3q27_bgk_lid.cpp) on liblbm_b200.  The loop body (stream, macros, lid and solid overwrites,
// equilibrium, BGK, bounce-back; :160-195) is one lbm_step call per reporting interval.  Same
// parameters as the reference (:60-80: 100^3, lid u = (0.1, 0, 0) on the z = nz-1 plane, Re 150,
// nu = u_lid nx / Re, 15,000 iterations) and the same start state (DENSITY = 1, U = 0 everywhere,
// :131-140), the reference's console report with the MLUPS formula corrected, no window.  Options:
//   --csv PATH    "Iterations,MLUPS" every 100 iterations
//   --dump PATH   final DENSITY, UX, UY, UZ as raw float64 [N | N | N | N], column-major
//
//   d3q27_bgk_lid [nx ny nz iterations] [--re R] [--u U] [--storage f32|f16s|bf16s]
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
    long long nx = 100, ny = 100, nz = 100, maxiter = 15000;
    double re = 150.0, ux_lid = 0.1;
    int storage = LBM_F32;
    std::string csv, dump;
    int pos = 0;
    for (int a = 1; a < argc; ++a) {
        const std::string s = argv[a];
        if (s == "--re" && a + 1 < argc) re = std::atof(argv[++a]);
        else if (s == "--u" && a + 1 < argc) ux_lid = std::atof(argv[++a]);
        else if (s == "--csv" && a + 1 < argc) csv = argv[++a];
        else if (s == "--dump" && a + 1 < argc) dump = argv[++a];
        else if (s == "--storage" && a + 1 < argc) {
            const std::string v = argv[++a];
            storage = v == "f16s" ? LBM_F16S : v == "bf16s" ? LBM_BF16S : LBM_F32;
        } else if (pos == 0) nx = std::atoll(s.c_str()), ++pos;
        else if (pos == 1) ny = std::atoll(s.c_str()), ++pos;
        else if (pos == 2) nz = std::atoll(s.c_str()), ++pos;
        else if (pos == 3) maxiter = std::atoll(s.c_str()), ++pos;
    }
    const long long total_nodes = nx * ny * nz;
    const double nu = ux_lid * nx / re;
    const double tau = 3.0 * nu + 0.5;
    const double omega = lbm_omega_from_re(ux_lid, (double)nx, re, 0);
    std::printf("LBM D3Q27 simulation\n");
    std::printf("Horizontal lid velocity ux_lid: %f\n", ux_lid);
    std::printf("Reynolds number: %f\n", re);
    std::printf("Lattice viscosity: %f\n", nu);
    std::printf("Relaxation time: %f\n", tau);
    std::printf("Relaxation parameter: %f\n", omega);

    lbm_desc d;
    lbm_desc_init(&d, LBM_D3Q27, LBM_BGK, storage, nx, ny, nz);
    d.omega = omega;
    std::vector<uint8_t> mask((size_t)total_nodes);
    if (lbm_setup_cavity3d(&d, mask.data(), ux_lid) != LBM_OK) return fail("lbm_setup_cavity3d");
    lbm_ctx* ctx = nullptr;
    if (lbm_create(&d, &ctx) != LBM_OK) return fail("lbm_create");
    if (lbm_init_equilibrium(ctx, nullptr, nullptr) != LBM_OK) return fail("lbm_init_equilibrium");

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
        std::vector<double> rho((size_t)total_nodes), u((size_t)(3 * total_nodes));
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
