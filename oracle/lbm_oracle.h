/*
 * lbm_oracle.h — CPU oracle for the LBM hot path.  TEST INFRASTRUCTURE ONLY: this code is the
 * checker for the CUDA engine (tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * it); the engine never links, loads or calls it.
 *
 * It restates the reference's per-iteration array program as plain per-cell loops:
 *   pull gather          cpp/d2q9_bgk_lid.cpp:18-28,86-87,124   (af::shift: out[x] = in[x - c], periodic)
 *   moments              cpp/d2q9_bgk_lid.cpp:131-138            (rho = sum F, u = sum(c F) / rho)
 *   boundary overwrites  cpp/d2q9_bgk_lid.cpp:141-146, cpp/d2q9_bgk_channel_packed.cpp:64-69
 *   BGK                  cpp/d2q9_bgk_lid.cpp:149-153, cpp/d3q27_bgk_lid.cpp:189-193
 *   MRT (dense 27x27)    rust/examples/d3q27_mrt_lid.rs:167-199,336-387
 *   bounce-back          cpp/d2q9_bgk_lid.cpp:97-98,126,155
 * Shan-Chen follows the published single-component model (Shan & Chen, Phys. Rev. E 47, 1815
 * (1993)): F = -G psi(x) sum_i w_i psi(x + c_i) c_i, u_eq = u + tau F / rho, psi = 1 - exp(-rho),
 * because the reference's cpp/d2q9_shanchen.cpp is an unfinished two-component draft.
 *
 * Parity status: the reference links ArrayFire (absent here), has no tests and no golden vectors,
 * so it cannot be run: parity unpinned against the reference itself.  The oracle is pinned to a
 * literal numpy emulation of the reference's array program (oracle/af_emulation.py) and to
 * invariants (rest state, conservation, symmetry).
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H
#include <stdint.h>

#define ORC_MAX_CLASSES 16
/* class flags: identical meaning to the engine's LBM_CELL_* (the mask format is shared) */
#define ORC_BOUNCE      0x01u
#define ORC_SET_RHO     0x02u
#define ORC_SET_UX      0x04u
#define ORC_SET_UY      0x08u
#define ORC_SET_UZ      0x10u
#define ORC_EQUILIBRIUM 0x20u
#define ORC_ZEROGRAD_XP 0x40u
#define ORC_ZOUHE_VEL_XM 0x80u
#define ORC_ZOUHE_RHO_XP 0x100u

typedef struct orc_desc {
    int32_t lattice;     /* 0 = D2Q9, 1 = D3Q27 */
    int32_t collision;   /* 0 = BGK, 1 = MRT, 2 = Shan-Chen */
    int32_t mrt_basis;   /* 0 = reference raw-monomial basis, 1 = Gram-Schmidt */
    int32_t n_classes;
    int64_t nx, ny, nz;
    double omega;
    double s[27];
    double G;
    uint32_t cls_flags[ORC_MAX_CLASSES];
    double cls_rho[ORC_MAX_CLASSES], cls_ux[ORC_MAX_CLASSES], cls_uy[ORC_MAX_CLASSES],
        cls_uz[ORC_MAX_CLASSES];
    const uint8_t* mask; /* N class ids or NULL */
} orc_desc;

/* Advance F (N*Q, layout [nx,ny,nz,Q]) by nsteps.  rho/u (N and dim*N, may be NULL) receive the
 * macroscopic fields the last step used.  threads <= 0: all OpenMP threads.  Returns 0 or -1. */
int orc_run_f64(const orc_desc* d, double* F, int64_t nsteps, double* rho, double* u, int threads);
int orc_run_f32(const orc_desc* d, float* F, int64_t nsteps, float* rho, float* u, int threads);
/* F = feq(rho, u) per cell (BGK equilibrium). rho may be NULL (=1), u may be NULL (=0). */
int orc_init_eq_f64(const orc_desc* d, double* F, const double* rho, const double* u);
/* Velocity set of the lattice; returns Q. */
int orc_velocities(int lattice, int* cx, int* cy, int* cz, double* w, int* opp);
/* The MRT matrices the oracle uses (row-major 27x27): M and its inverse. */
int orc_mrt_matrices(int basis, double* M, double* Minv);
/* FP64 sums of F: mass and momentum. */
void orc_sums_f64(const orc_desc* d, const double* F, double out[4]);
#endif
