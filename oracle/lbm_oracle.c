/*
 * lbm_oracle.c — CPU oracle for the LBM hot path (TEST INFRASTRUCTURE; see lbm_oracle.h).
 * Plain C + OpenMP, FP64 and FP32 instantiations of one step routine (oracle_step.inc).
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* D2Q9 velocity set, weights and opposites: cpp/d2q9_bgk_lid.cpp:72-84 */
static const int D2_CX[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
static const int D2_CY[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
static const double D2_W[9] = {4. / 9., 1. / 9., 1. / 9., 1. / 9., 1. / 9.,
                               1. / 36., 1. / 36., 1. / 36., 1. / 36.};
/* opposite map built from nb_index_arr {2,3,0,1,6,7,4,5} over directions 1..8 (:82) */
static const int D2_OPP[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};

/* D3Q27: cpp/d3q27_bgk_lid.cpp:98-113 */
static const int D3_CX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1,
                              0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
static const int D3_CY[27] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0,
                              1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1};
static const int D3_CZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1,
                              1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1};
static const double D3_W[27] = {
    8. / 27.,  2. / 27.,  2. / 27.,  2. / 27.,  2. / 27.,  2. / 27.,  2. / 27.,
    1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,
    1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,  1. / 216., 1. / 216.,
    1. / 216., 1. / 216., 1. / 216., 1. / 216., 1. / 216., 1. / 216.};
/* nb_index_arr {1,0,3,2,5,4,9,8,7,6,13,12,11,10,17,16,15,14,25,24,23,22,21,20,19,18} (:111), +1 shifted */
static const int D3_OPP[27] = {0,  2,  1,  4,  3,  6,  5,  10, 9,  8,  7,  14, 13, 12,
                               11, 18, 17, 16, 15, 26, 25, 24, 23, 22, 21, 20, 19};

int orc_velocities(int lattice, int* cx, int* cy, int* cz, double* w, int* opp) {
    int q = lattice == 0 ? 9 : 27;
    for (int i = 0; i < q; ++i) {
        if (cx) cx[i] = lattice == 0 ? D2_CX[i] : D3_CX[i];
        if (cy) cy[i] = lattice == 0 ? D2_CY[i] : D3_CY[i];
        if (cz) cz[i] = lattice == 0 ? 0 : D3_CZ[i];
        if (w) w[i] = lattice == 0 ? D2_W[i] : D3_W[i];
        if (opp) opp[i] = lattice == 0 ? D2_OPP[i] : D3_OPP[i];
    }
    return q;
}

/* ---- MRT matrices ------------------------------------------------------------------------
 * Reference basis rows: rust/examples/d3q27_mrt_lid.rs:167-193 (row 0 = all ones, rows 1..26 as
 * set_row lists them).  Built densely here; the engine uses a factorised form instead.          */
static void mrt_reference_rows(double M[27][27]) {
    for (int i = 0; i < 27; ++i) {
        double x = D3_CX[i], y = D3_CY[i], z = D3_CZ[i];
        double r[27] = {1.0,
                        x,
                        y,
                        z,
                        x * y,
                        x * z,
                        y * z,
                        x * x + y * y + z * z,
                        x * x - y * y,
                        x * x - z * z,
                        x * y * y,
                        x * z * z,
                        y * x * x,
                        z * x * x,
                        y * z * z,
                        z * y * y,
                        x * y * z,
                        x * x * y * y,
                        x * x * z * z,
                        y * y * z * z,
                        x * x * y * z,
                        x * y * y * z,
                        x * y * z * z,
                        x * y * y * z * z,
                        x * x * y * z * z,
                        x * x * y * y * z,
                        x * x * y * y * z * z};
        for (int k = 0; k < 27; ++k) M[k][i] = r[k];
    }
}

/* Classical Gram-Schmidt of the reference rows, in row order, unweighted inner product. */
static void mrt_gram_schmidt_rows(double M[27][27]) {
    double R[27][27];
    mrt_reference_rows(R);
    for (int k = 0; k < 27; ++k) {
        double v[27];
        for (int i = 0; i < 27; ++i) v[i] = R[k][i];
        for (int j = 0; j < k; ++j) {
            double num = 0, den = 0;
            for (int i = 0; i < 27; ++i) {
                num += R[k][i] * M[j][i];
                den += M[j][i] * M[j][i];
            }
            for (int i = 0; i < 27; ++i) v[i] -= num / den * M[j][i];
        }
        for (int i = 0; i < 27; ++i) M[k][i] = fabs(v[i]) < 1e-12 ? 0.0 : v[i];
    }
}

/* Gauss-Jordan inverse with partial pivoting (FP64). Returns 0 on success. */
static int invert27(double A_in[27][27], double Ainv[27][27]) {
    double A[27][54];
    for (int i = 0; i < 27; ++i)
        for (int j = 0; j < 54; ++j) A[i][j] = j < 27 ? A_in[i][j] : (j - 27 == i ? 1.0 : 0.0);
    for (int c = 0; c < 27; ++c) {
        int p = c;
        for (int r = c + 1; r < 27; ++r)
            if (fabs(A[r][c]) > fabs(A[p][c])) p = r;
        if (fabs(A[p][c]) < 1e-12) return -1;
        if (p != c)
            for (int j = 0; j < 54; ++j) {
                double t = A[c][j];
                A[c][j] = A[p][j];
                A[p][j] = t;
            }
        double piv = A[c][c];
        for (int j = 0; j < 54; ++j) A[c][j] /= piv;
        for (int r = 0; r < 27; ++r) {
            if (r == c || A[r][c] == 0.0) continue;
            double f = A[r][c];
            for (int j = 0; j < 54; ++j) A[r][j] -= f * A[c][j];
        }
    }
    for (int i = 0; i < 27; ++i)
        for (int j = 0; j < 27; ++j) Ainv[i][j] = A[i][j + 27];
    return 0;
}

int orc_mrt_matrices(int basis, double* Mout, double* Minv_out) {
    double M[27][27], Mi[27][27];
    if (basis == 0)
        mrt_reference_rows(M);
    else
        mrt_gram_schmidt_rows(M);
    if (invert27(M, Mi) != 0) return -1;
    if (Mout) memcpy(Mout, M, sizeof(M));
    if (Minv_out) memcpy(Minv_out, Mi, sizeof(Mi));
    return 0;
}

static int resolve_threads(int threads) {
#ifdef _OPENMP
    return threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

/* ---- FP64 and FP32 step routines ---------------------------------------------------------- */
#define REAL double
#define SFX(name) name##_f64
#define EXPR exp
#include "oracle_step.inc"
#undef REAL
#undef SFX
#undef EXPR

#define REAL float
#define SFX(name) name##_f32
#define EXPR expf
#include "oracle_step.inc"
#undef REAL
#undef SFX
#undef EXPR

int orc_init_eq_f64(const orc_desc* d, double* F, const double* rho, const double* u) {
    int cx[27], cy[27], cz[27], opp[27];
    double w[27];
    int q = orc_velocities(d->lattice, cx, cy, cz, w, opp);
    int64_t N = d->nx * d->ny * d->nz;
    int dim = d->lattice == 0 ? 2 : 3;
    for (int64_t c = 0; c < N; ++c) {
        double r = rho ? rho[c] : 1.0;
        double ux = u ? u[c] : 0.0, uy = u ? u[N + c] : 0.0, uz = (u && dim == 3) ? u[2 * N + c] : 0.0;
        double usq = ux * ux + uy * uy + uz * uz;
        for (int i = 0; i < q; ++i) {
            double eu = cx[i] * ux + cy[i] * uy + cz[i] * uz;
            F[c + N * i] = w[i] * r * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * usq);
        }
    }
    return 0;
}

void orc_sums_f64(const orc_desc* d, const double* F, double out[4]) {
    int cx[27], cy[27], cz[27];
    int q = orc_velocities(d->lattice, cx, cy, cz, NULL, NULL);
    int64_t N = d->nx * d->ny * d->nz;
    double m = 0, jx = 0, jy = 0, jz = 0;
    for (int i = 0; i < q; ++i) {
        double s = 0;
        for (int64_t c = 0; c < N; ++c) s += F[c + N * i];
        m += s;
        jx += cx[i] * s;
        jy += cy[i] * s;
        jz += cz[i] * s;
    }
    out[0] = m;
    out[1] = jx;
    out[2] = jy;
    out[3] = jz;
}
