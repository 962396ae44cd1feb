// d3q27_mrt_lid.cpp — headless version of the reference's D3Q27 MRT lid-driven cavity
// (rust/examples/d3q27_mrt_lid.rs; cpp/d3q27_mrt_lid.cpp has a singular moment matrix) on
// liblbm_b200.  The reference's loop body (stream, macros, lid/solid overwrites, m = F M^T, relax to
// meq, F = m* M^-T, bounce-back; :304-389) is one lbm_step call per reporting interval.  Start state
// as the reference: uniform 1/27 collided once towards meq(rho = 1, u = 0) (:228-287).  Console report
// as the reference (:147-149, :390-402) with the MLUPS formula corrected; optional outputs:
//   --csv PATH    "Iterations,MLUPS" every 100 iterations
//   --dump PATH   final DENSITY, UX, UY, UZ as raw float64 [N | N | N | N], column-major
//
//   d3q27_mrt_lid [n iterations] [--u U] [--storage f32|f16s|bf16s] [--gram-schmidt --re R]
// Default: the reference's rates and raw-monomial basis; --gram-schmidt takes the benchmark form
// (Gram-Schmidt basis, shear rate from Re on n, other rates 1.2).
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
    long long n = 64, maxiter = 1000;
    double ux_lid = 0.05, re = 1000.0;
    int storage = LBM_F32;
    bool gs = false;
    std::string csv, dump;
    int pos = 0;
    for (int a = 1; a < argc; ++a) {
        const std::string s = argv[a];
        if (s == "--u" && a + 1 < argc) ux_lid = std::atof(argv[++a]);
        else if (s == "--re" && a + 1 < argc) re = std::atof(argv[++a]);
        else if (s == "--csv" && a + 1 < argc) csv = argv[++a];
        else if (s == "--dump" && a + 1 < argc) dump = argv[++a];
        else if (s == "--gram-schmidt") gs = true;
        else if (s == "--storage" && a + 1 < argc) {
            const std::string v = argv[++a];
            storage = v == "f16s" ? LBM_F16S : v == "bf16s" ? LBM_BF16S : LBM_F32;
        } else if (pos == 0) n = std::atoll(s.c_str()), ++pos;
        else if (pos == 1) maxiter = std::atoll(s.c_str()), ++pos;
    }
    const long long total_nodes = n * n * n;
    lbm_desc d;
    lbm_desc_init(&d, LBM_D3Q27, LBM_MRT, storage, n, n, n);
    double sv;
    if (gs) {
        sv = 1.0 / (3.0 * (ux_lid * n / re) + 0.5);
        lbm_mrt_rates(d.mrt_s, sv, 1.2);
        d.mrt_basis = LBM_MRT_GRAM_SCHMIDT;
    } else {
        lbm_mrt_reference_rates(d.mrt_s);
        sv = d.mrt_s[4];
        d.mrt_basis = LBM_MRT_REF;
    }
    const double sb = d.mrt_s[7];
    std::printf("LBM D3Q27 MRT simulation\n");
    std::printf("Lid speed: %f\n", ux_lid);
    std::printf("Lattice viscosity: %f\n", (1.0 / sv - 0.5) / 3.0);
    std::printf("Bulk viscosity: %f\n", (2.0 / 3.0) * (1.0 / sb - 0.5) / 3.0);

    std::vector<uint8_t> mask((size_t)total_nodes);
    if (lbm_setup_cavity3d(&d, mask.data(), ux_lid) != LBM_OK) return fail("lbm_setup_cavity3d");
    lbm_ctx* ctx = nullptr;
    if (lbm_create(&d, &ctx) != LBM_OK) return fail("lbm_create");
    // start state: uniform 1/27 collided once towards meq(1, 0), the same in every cell
    double f_in[27], f0[27];
    for (double& v : f_in) v = 1.0 / 27.0;
    const double u0[3] = {0.0, 0.0, 0.0};
    if (lbm_mrt_collide_host(&d, f_in, 1.0, u0, f0) != LBM_OK) return fail("lbm_mrt_collide_host");
    {
        std::vector<double> F((size_t)(27 * total_nodes));
        for (int i = 0; i < 27; ++i)
            for (long long c = 0; c < total_nodes; ++c) F[(size_t)(i * total_nodes + c)] = f0[i];
        if (lbm_set_populations(ctx, F.data(), LBM_DTYPE_F64, LBM_HOST) != LBM_OK) return fail("lbm_set_populations");
    }
    if (lbm_sync(ctx) != LBM_OK) return fail("lbm_sync");

    FILE* fcsv = csv.empty() ? nullptr : std::fopen(csv.c_str(), "w");
    if (fcsv) std::fprintf(fcsv, "Iterations,MLUPS\n");
    const auto t0 = std::chrono::steady_clock::now();
    long long iter = 0;
    while (iter < maxiter) {
        const long long k = std::min<long long>(100 - iter % 100, maxiter - iter);
        if (lbm_step(ctx, k) != LBM_OK) return fail("lbm_step");
        iter += k;
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
