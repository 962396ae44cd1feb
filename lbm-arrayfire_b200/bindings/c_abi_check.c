/* c_abi_check.c — a plain C99 caller of liblbm_b200 (no C++), built with gcc against include/lbm.h.
 *
 *   c_abi_check layout      prints the size of lbm_cell_class / lbm_desc and the offset of every field
 *                           ("name value" lines); bindings/lbm_sys.rs asserts the same numbers for its
 *                           #[repr(C)] mirrors, and tests/test_bindings.py compares the two
 *   c_abi_check run N S     D2Q9 lid cavity N x N (lid 0.1, Re 100, the C++ viscosity rule), S steps
 *                           through the C ABI; prints the FP64 mass and momentum sums ("sums m jx jy")
 *                           and the status of every call (needs a B200)                              */
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>

#include "lbm.h"

#define FIELD(T, f) printf("offsetof " #T "." #f " %zu\n", offsetof(T, f))

static int layout(void) {
    printf("sizeof lbm_cell_class %zu\n", sizeof(lbm_cell_class));
    FIELD(lbm_cell_class, flags);
    FIELD(lbm_cell_class, reserved);
    FIELD(lbm_cell_class, rho);
    FIELD(lbm_cell_class, ux);
    FIELD(lbm_cell_class, uy);
    FIELD(lbm_cell_class, uz);
    printf("sizeof lbm_desc %zu\n", sizeof(lbm_desc));
    FIELD(lbm_desc, lattice);
    FIELD(lbm_desc, collision);
    FIELD(lbm_desc, storage);
    FIELD(lbm_desc, mrt_basis);
    FIELD(lbm_desc, arithmetic);
    FIELD(lbm_desc, rounding);
    FIELD(lbm_desc, nx);
    FIELD(lbm_desc, ny);
    FIELD(lbm_desc, nz);
    FIELD(lbm_desc, omega);
    FIELD(lbm_desc, mrt_s);
    FIELD(lbm_desc, sc_G);
    FIELD(lbm_desc, storage_scale);
    FIELD(lbm_desc, n_classes);
    FIELD(lbm_desc, device);
    FIELD(lbm_desc, classes);
    FIELD(lbm_desc, mask);
    printf("abi_version %d\n", lbm_abi_version());
    return 0;
}

static int check(int rc, const char* what) {
    if (rc != LBM_OK) fprintf(stderr, "%s: %s (%s)\n", what, lbm_strerror(rc), lbm_last_error());
    return rc;
}

static int run(long long n, long long steps) {
    lbm_desc d;
    lbm_desc_init(&d, LBM_D2Q9, LBM_BGK, LBM_F32, n, n, 1);
    d.omega = lbm_omega_from_re(0.1, (double)n, 100.0, 0);
    unsigned char* mask = (unsigned char*)malloc((size_t)(n * n));
    if (!mask) return 1;
    if (check(lbm_setup_cavity2d(&d, mask, 0.1), "lbm_setup_cavity2d")) return 1;
    lbm_ctx* ctx = NULL;
    if (check(lbm_create(&d, &ctx), "lbm_create")) return 1;
    double s[4];
    int rc = check(lbm_step(ctx, steps), "lbm_step");
    if (!rc) rc = check(lbm_sync(ctx), "lbm_sync");
    if (!rc) rc = check(lbm_sums_fp64(ctx, s), "lbm_sums_fp64");
    if (!rc) printf("sums %.17g %.17g %.17g\n", s[0], s[1], s[2]);
    printf("steps_done %lld\n", (long long)lbm_steps_done(ctx));
    lbm_destroy(ctx);
    free(mask);
    return rc ? 1 : 0;
}

int main(int argc, char** argv) {
    if (argc > 1 && argv[1][0] == 'l') return layout();
    if (argc > 3 && argv[1][0] == 'r') return run(atoll(argv[2]), atoll(argv[3]));
    fprintf(stderr, "usage: c_abi_check layout | run N STEPS\n");
    return 2;
}
