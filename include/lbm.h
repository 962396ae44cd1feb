/*
 * lbm.h — C ABI of the B200-native Lattice Boltzmann engine (liblbm_b200.so).
 *
 * One lbm_step() call advances the populations by whole time steps with one fused
 * sm_100a kernel per step (pull streaming + BGK/MRT/Shan-Chen collision + cell-class
 * boundary handling).  It replaces the body of the reference's time loop: everything from
 *   F_streamed = F(nb_index)            (cpp/d2q9_bgk_lid.cpp:124)
 * to
 *   F(REFLECTED) = BOUNCEDBACK           (cpp/d2q9_bgk_lid.cpp:155)
 * and the same span in cpp/d2q9_bgk_channel_packed.cpp:54-74, cpp/d3q27_bgk_lid.cpp:160-195,
 * rust/examples/d2q9_bgk_lid.rs:153-191 and rust/examples/d3q27_mrt_lid.rs:304-389.
 *
 * Conventions kept from the reference:
 *  - population layout: column-major [nx, ny(, nz), Q], i.e. F[x + nx*(y + ny*(z + nz*i))]
 *    (moddims(range(N*Q), nx, ny, 9) at cpp/d2q9_bgk_lid.cpp:86);
 *  - velocity ordering and weights: D2Q9 cpp/d2q9_bgk_lid.cpp:72-79, D3Q27 cpp/d3q27_bgk_lid.cpp:98-107;
 *  - opposite-direction map: cpp/d2q9_bgk_lid.cpp:82, cpp/d3q27_bgk_lid.cpp:111;
 *  - periodic wrap of the pull gather (af::shift semantics, out[x] = in[x - c]);
 *  - full-way bounce-back: a solid cell stores the reversed streamed populations after the
 *    collision (cpp/d2q9_bgk_lid.cpp:97-98,126,155);
 *  - boundary conditions as overwrites of rho/u before the equilibrium (cpp/d2q9_bgk_lid.cpp:141-146).
 *
 * Errors: every int-returning call returns LBM_OK (0) or a negative LBM_ERR_* code; no C++
 * exception crosses this boundary (the reference's catch(af::exception) at cpp/d2q9_bgk_lid.cpp:219).
 * lbm_last_error() gives a message for the last failing call on the calling thread.
 * Threading: one context per host thread at a time; calls on one context are not thread-safe.
 * Ownership: the context owns its device buffers; host pointers are borrowed for the call only.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------------------------- */
#define LBM_OK               0
#define LBM_ERR_INVALID    (-1)  /* bad argument or descriptor field */
#define LBM_ERR_CUDA       (-2)  /* a CUDA runtime call failed */
#define LBM_ERR_NOMEM      (-3)  /* device or host allocation failed */
#define LBM_ERR_DIVERGED   (-4)  /* NaN/Inf found in the populations */
#define LBM_ERR_UNSUPPORTED (-5) /* combination not built (e.g. MRT on D2Q9) */
#define LBM_ERR_NO_DEVICE  (-6)  /* no CUDA device / not an sm_100 device */
#define LBM_ERR_STATE      (-7)  /* call not valid in the current state */
#define LBM_ERR_TIMEOUT    (-8)  /* a bounded device-side wait gave up (the step kernel returned early) */

/* ---- enumerations ---------------------------------------------------------------------- */
enum lbm_lattice   { LBM_D2Q9 = 0, LBM_D3Q27 = 1 };
enum lbm_collision { LBM_BGK = 0, LBM_MRT = 1, LBM_SHANCHEN = 2 };
/* Storage of the populations in HBM.  Arithmetic is FP32 for F32/F16S/BF16S and FP64 for F64.
 * F16S / BF16S hold the shifted population (f_i - w_i) * storage_scale in 16 bits.            */
enum lbm_storage   { LBM_F32 = 0, LBM_F16S = 1, LBM_BF16S = 2, LBM_F64 = 3 };
/* MRT moment basis.  REF: the raw-monomial 27x27 matrix of rust/examples/d3q27_mrt_lid.rs:167-193
 * with its equilibrium-moment table (:357-383).  GRAM_SCHMIDT: the same rows orthogonalised in order
 * (unweighted inner product over the 27 velocities), equilibrium moments = M * feq(rho,u).       */
enum lbm_mrt_basis { LBM_MRT_REF = 0, LBM_MRT_GRAM_SCHMIDT = 1 };
/* How the step arithmetic treats the populations.
 * DEVIATION (default): every kernel computes on d_i = f_i - w_i (moments, equilibrium, MRT
 *   transform); rho = 1 + sum d.  More accurate in FP32 than the reference: no cancellation of the
 *   O(w) parts and no systematic density drift.  Required for F16S/BF16S storage.
 * ABSOLUTE: the reference's arithmetic on the populations themselves (rho = sum f,
 *   F = omega FEQ + (1 - omega) F_streamed, cpp/d2q9_bgk_lid.cpp:131-153), so FP32 results carry the
 *   same rounding behaviour as the reference's FP32 runs.  BGK and Shan-Chen, F32 or F64 storage,
 *   single lattices (MRT always uses DEVIATION: its factorised transform cannot reproduce the
 *   rounding of the reference's dense FP32 GEMMs anyway).                                        */
enum lbm_arithmetic { LBM_ARITH_DEVIATION = 0, LBM_ARITH_ABSOLUTE = 1 };
/* How F16S / BF16S storage rounds the collided populations.
 * STOCHASTIC (default): unbiased stochastic rounding (sm_100a cvt.rs) with random words hashed from the
 *   cell index and the step number -- deterministic and the same in every kernel family, graph or not.
 *   Round-to-nearest repeats the same error every step where a flow is (nearly) steady, and slow modes
 *   integrate that bias: on the D3Q27 MRT 256^3 cavity it left 1.3e-3 rel. L2 velocity error against FP64
 *   after 5,000 steps, and the Shan-Chen 1024^2 BF16S run lost 4 % of its mass in 20,000 steps.
 * NEAREST: round to nearest even.  F32/F64 storage ignores the field.                               */
enum lbm_rounding  { LBM_ROUND_STOCHASTIC = 0, LBM_ROUND_NEAREST = 1 };
/* Host buffer element type for population / field transfers. */
enum lbm_dtype     { LBM_DTYPE_F32 = 0, LBM_DTYPE_F64 = 1 };
/* Where a transfer buffer lives. */
enum lbm_memory    { LBM_HOST = 0, LBM_DEVICE = 1 };

/* ---- cell classes ------------------------------------------------------------------------
 * The mask holds one uint8 class id per cell (column-major like the populations).  Each class
 * states what happens to a cell of that class in every step.  Class 0 is plain fluid unless
 * the descriptor redefines it.  The flags reproduce the reference's boundary overwrites:
 *   solid (ON list):   BOUNCE|SET_RHO|SET_UX|SET_UY|SET_UZ with rho=u=0  (cpp/d2q9_bgk_lid.cpp:144-146,155)
 *   lid row:           SET_UX|SET_UY(|SET_UZ) with the lid velocity   (cpp/d2q9_bgk_lid.cpp:141-142)
 *   channel inlet:     SET_UX|SET_RHO, rho=1                          (cpp/d2q9_bgk_channel_packed.cpp:64,68)
 *   channel outlet:    SET_RHO, rho=1                                 (cpp/d2q9_bgk_channel_packed.cpp:69)     */
#define LBM_MAX_CLASSES 16
#define LBM_CELL_BOUNCE       0x01u /* store reversed streamed populations (i>=1) after collision  */
#define LBM_CELL_SET_RHO      0x02u /* overwrite rho with class rho before the equilibrium         */
#define LBM_CELL_SET_UX       0x04u /* overwrite u_x                                                */
#define LBM_CELL_SET_UY       0x08u /* overwrite u_y                                                */
#define LBM_CELL_SET_UZ       0x10u /* overwrite u_z (D3Q27)                                        */
#define LBM_CELL_EQUILIBRIUM  0x20u /* write feq(rho,u) for every direction (Dirichlet equilibrium) */
#define LBM_CELL_ZEROGRAD_XP  0x40u /* outlet on the x = nx-1 face: populations arriving from +x are
                                       copied from the streamed state of cell x-1 (zero gradient)  */
/* Zou-He open boundaries (Zou & He 1997; no counterpart in the reference, whose only open boundaries
 * are the density/velocity overwrites above).  D2Q9 BGK only.  Before the collision the populations
 * that arrive from outside the lattice are rebuilt from the known ones so that the cell has the
 * prescribed velocity or density; the collision then proceeds as for fluid.                       */
#define LBM_CELL_ZOUHE_VEL_XM 0x80u /* velocity inlet on the x = 0 face: class (ux, uy) prescribed,
                                       rho and the populations with c_x = +1 follow               */
#define LBM_CELL_ZOUHE_RHO_XP 0x100u /* pressure outlet on the x = nx-1 face: class rho and uy
                                       prescribed, ux and the populations with c_x = -1 follow     */

typedef struct lbm_cell_class {
    uint32_t flags;
    uint32_t reserved;      /* 0 */
    double rho, ux, uy, uz; /* used in FP64 by F64 storage, rounded to FP32 otherwise */
} lbm_cell_class;

/* ---- lattice descriptor ------------------------------------------------------------------ */
typedef struct lbm_desc {
    int32_t lattice;        /* enum lbm_lattice                                               */
    int32_t collision;      /* enum lbm_collision                                             */
    int32_t storage;        /* enum lbm_storage                                               */
    int32_t mrt_basis;      /* enum lbm_mrt_basis (MRT only)                                  */
    int32_t arithmetic;     /* enum lbm_arithmetic                                            */
    int32_t rounding;       /* enum lbm_rounding (16-bit storage)                             */
    int64_t nx, ny, nz;     /* nz = 1 for D2Q9                                                */
    double omega;           /* BGK / Shan-Chen relaxation 1/tau                               */
    double mrt_s[27];       /* MRT relaxation rate per moment row (rust/examples/d3q27_mrt_lid.rs:122-150) */
    double sc_G;            /* Shan-Chen interaction strength; psi = 1 - exp(-rho)            */
    double storage_scale;   /* F16S/BF16S: stored = (f - w) * scale; 0 selects the default    */
    int32_t n_classes;      /* entries used in classes[] (>= 1)                               */
    int32_t device;         /* CUDA device ordinal                                            */
    lbm_cell_class classes[LBM_MAX_CLASSES];
    const uint8_t* mask;    /* host, N class ids column-major; NULL = every cell class 0      */
} lbm_desc;

typedef struct lbm_ctx lbm_ctx;
typedef struct lbm_batch lbm_batch;

/* ---- library --------------------------------------------------------------------------- */
int         lbm_abi_version(void);
const char* lbm_strerror(int status);
const char* lbm_last_error(void);
/* Fill a descriptor with defaults: fluid class 0, omega 1, MRT rates 1, device 0. */
void        lbm_desc_init(lbm_desc* d, int lattice, int collision, int storage,
                          int64_t nx, int64_t ny, int64_t nz);
int         lbm_q(int lattice);                          /* 9 or 27 */
/* Velocity set and weights exactly as the reference lists them (a1 of the path). */
int         lbm_velocities(int lattice, int32_t* cx, int32_t* cy, int32_t* cz, double* w, int32_t* opp);

/* ---- single lattice ---------------------------------------------------------------------
 * lbm_create: validates the descriptor, allocates two population buffers (ping-pong) plus the mask
 * on the device, and sets every population to feq(rho=1, u=0) of each cell's class values.       */
int  lbm_create(const lbm_desc* d, lbm_ctx** out);
void lbm_destroy(lbm_ctx* c);
/* Populations in the reference layout [nx,ny(,nz),Q].  src/dst: host or device pointer. */
int  lbm_set_populations(lbm_ctx* c, const void* src, int dtype, int memory);
int  lbm_get_populations(lbm_ctx* c, void* dst, int dtype, int memory);
/* F = feq(rho, u) per cell, the reference's start state (cpp/d2q9_bgk_lid.cpp:100-107).
 * rho: N doubles or NULL (=1); u: dim*N doubles [ux | uy (| uz)] or NULL (=0).  Host pointers. */
int  lbm_init_equilibrium(lbm_ctx* c, const double* rho, const double* u);
/* Advance nsteps time steps, asynchronously on the context stream. */
int  lbm_step(lbm_ctx* c, int64_t nsteps);
/* Wait for the context's stream; returns LBM_ERR_TIMEOUT if a step kernel gave up a bounded wait. */
int  lbm_sync(lbm_ctx* c);
/* Macroscopic fields the last step's collision used, after the class overwrites (the reference's
 * DENSITY / UX / UY / UZ after an iteration).  Before any step: moments of the current populations.
 * rho: N values; u: dim*N values [ux | uy (| uz)]. Either may be NULL.                            */
int  lbm_get_macros(lbm_ctx* c, void* rho, void* u, int dtype, int memory);
/* FP64 sums over all cells of the current populations: out[0] = mass, out[1..3] = momentum.
 * Returns LBM_ERR_DIVERGED when a population is NaN or Inf.                                       */
int  lbm_sums_fp64(lbm_ctx* c, double out[4]);
/* Steady-state residual in FP64: sqrt(sum |u_t - u_{t-1}|^2 / sum |u_t|^2) over class-0 cells. */
int  lbm_residual_fp64(lbm_ctx* c, double* out);
/* Device time of the most recent lbm_step call in milliseconds (CUDA events on the context stream). */
int  lbm_last_step_ms(lbm_ctx* c, float* ms);
int64_t lbm_steps_done(const lbm_ctx* c);
/* The context's CUDA stream (cudaStream_t) and device buffers, for callers that interoperate. */
void* lbm_stream(lbm_ctx* c);
/* NULL restores the context's own (non-blocking) stream; the legacy default stream is cudaStreamLegacy. */
int   lbm_set_stream(lbm_ctx* c, void* stream);
/* Current population buffer on the device (storage type of the descriptor) and its byte size. */
void* lbm_device_populations(lbm_ctx* c, size_t* bytes);
int   lbm_get_desc(const lbm_ctx* c, lbm_desc* out);
/* Faces of the slowest axis (z planes of D3Q27, y rows of D2Q9) for halo exchanges between slabs of
 * one lattice (no counterpart in the reference, which runs on one device): the populations of
 * directions dirs[0..ndirs) on plane `plane` of the current buffer, packed [ndirs][plane cells] as
 * stored words (the descriptor's storage type, no conversion, so an exchange is bit-exact).
 * memory = LBM_DEVICE: asynchronous on the context stream; LBM_HOST: returns when the copy is done. */
int   lbm_face_get(lbm_ctx* c, int64_t plane, const int32_t* dirs, int32_t ndirs, void* dst, int memory);
int   lbm_face_set(lbm_ctx* c, int64_t plane, const int32_t* dirs, int32_t ndirs, const void* src, int memory);
/* One time step over planes first + k * stride, k < count, of the slowest axis only (z planes of D3Q27,
 * y rows of D2Q9), from the current buffer into the other one, in one launch, asynchronously on
 * `stream` (a cudaStream_t; NULL: the context stream).  Calls for disjoint plane sets that together
 * cover every plane make one step; the last of them passes finish = 1, which makes the written buffer
 * current.  Calls on different streams may run at the same time (they read one buffer and write
 * disjoint planes of the other); the caller orders every one of them before the next step's first
 * launch.  This lets a slab of a decomposed lattice update its two boundary planes (first 1, count 2,
 * stride n - 1) and exchange their faces on a side stream while its interior planes are updated (no
 * counterpart in the reference).  Shan-Chen plane sets run the one-pass window kernel (bit-identical
 * to the two passes; it writes psi of its own rows only).  Planes outside the sets keep whatever the
 * other buffer held.                                                                               */
int   lbm_step_planes(lbm_ctx* c, int64_t first, int64_t count, int64_t stride, int finish, void* stream);
/* Splits the SMs between the context stream and side streams for the row pipeline's persistent grid
 * (0..64; default 0): its launches on the context stream leave `sms` SMs free, so that kernels on
 * another stream (a face exchange, a collective) run beside a step instead of after it, and its
 * lbm_step_planes launches on another stream use at most those `sms` SMs (with sms > 0).            */
int   lbm_set_reserved_sms(lbm_ctx* c, int sms);
/* Both population buffers: the current one and the one the next step writes (device pointers). */
int   lbm_device_buffers(lbm_ctx* c, void** current, void** next, size_t* bytes);
/* Index of this lattice's first cell within a larger lattice it is a part of (a slab of a decomposed
 * lattice; any integer, taken modulo 2^32; default 0).  Stochastic rounding hashes that global index
 * with the step number, so the slabs of a decomposed lattice round exactly like the undivided lattice.
 * No counterpart in the reference (one lattice on one device).                                     */
int   lbm_set_cell_offset(lbm_ctx* c, int64_t offset);
/* Block width (threads along x) used by the step kernel; 0 = autotune on first step. */
int   lbm_set_block(lbm_ctx* c, int threads_x);
int   lbm_get_block(const lbm_ctx* c);
/* Step-kernel family.  PLAIN: one thread per cell, populations read straight from HBM.  ROWS
 * (D3Q27 BGK/MRT or D2Q9 BGK, deviation arithmetic, F32/F16S/BF16S, nx >= 32 a multiple of 16):
 * groups of whole rows (segments of rows wider than 1024 cells) staged in shared memory by bulk
 * copies (TMA) through an mbarrier ring; for D2Q9 Shan-Chen (any shape and storage) the one-pass
 * kernel (a window sliding down y: psi of the next row into a shared ring, the force from it) instead
 * of the two passes of PLAIN.  CLUSTER (D2Q9 BGK, deviation arithmetic, both buffers within the
 * shared memory of one thread-block cluster: 128^2 FP32, 256^2 FP16S): the lattice stays resident in
 * the cluster's shared memory for up to 4096 steps of one launch, one cluster barrier per step, for
 * lattices too small to fill the GPU (a step is then launch-bound); lbm_step_planes and lone steps
 * inside CUDA graphs take PLAIN.  AUTO (default): the autotuner times the eligible ones.  All give
 * bit-identical results.                                                                            */
enum lbm_kernel { LBM_KERNEL_AUTO = 0, LBM_KERNEL_PLAIN = 1, LBM_KERNEL_ROWS = 2, LBM_KERNEL_CLUSTER = 3 };
int   lbm_set_kernel(lbm_ctx* c, int kind);
int   lbm_get_kernel(const lbm_ctx* c);              /* the family in use (PLAIN, ROWS or CLUSTER), or AUTO before the first step */

/* ---- test hook of the bounded device-side waits (no counterpart in the reference) --------
 * Arms a one-shot stall of the row pipeline so that tests can drive its bounded mbarrier waits to
 * their limit without any fault: the next lbm_step launches its first step on its own, the producer
 * of that launch issues no copies for work item `item` (a row group or row segment in the order the
 * persistent CTAs take them; item 0 is the first stage of CTA 0), and every wait of that launch gives
 * up after `wait_clocks` SM clocks (2^10 .. 2^32; 2^21 is about a millisecond).  The consumers waiting
 * for that stage time out, then its producer; the launch returns and lbm_sync reports LBM_ERR_TIMEOUT
 * once (it clears the error word).  The populations written by that step are invalid: set or
 * re-initialise them before stepping on.  Needs lbm_set_kernel(c, LBM_KERNEL_ROWS) (BGK or MRT).   */
int  lbm_test_stall_next_step(lbm_ctx* c, int64_t item, int64_t wait_clocks);
/* Test hook (no counterpart in the reference): on = 1 makes the plain step kernels and the one-pass
 * Shan-Chen kernel index populations in 64 bits even where 32-bit indices suffice (they take 32-bit
 * ones on lattices with Q N <= 2^32), so that tests can compare both forms bit for bit on small
 * lattices; on = 0 restores the choice.                                                           */
int  lbm_test_index64(lbm_ctx* c, int on);

/* ---- conservation sums without allocation -----------------------------------------------
 * No counterpart in the reference.  For callers that cannot let a library call cudaMalloc or
 * cudaFree — applications whose device memory belongs to another allocator (a framework's caching
 * allocator, a pool reserved up front), where an extra cudaMalloc can fail or fragment the pool and a
 * cudaFree synchronises the whole device.  Computes the same FP64 mass/momentum sums as
 * lbm_sums_fp64, over a caller-owned population buffer on the current device (the engine's storage
 * format and layout, e.g. from lbm_device_populations), with no allocation of any kind: the scratch
 * (one partial per block + the result) is a fixed array in the library's device image, held by every
 * GPU that loads the library until the process exits (640 KB).
 *  - At most LBM_NOALLOC_MAX_CELLS cells (nx * ny * nz, bounded without overflow); larger lattices
 *    are rejected with LBM_ERR_INVALID.
 *  - Every call looks up the array's device address on the current device (cudaGetSymbolAddress,
 *    which allocates nothing); the first call on a device may load the library's device code, so make
 *    that first call before any stream capture.
 *  - Every call shares the one array, so calls that overlap on the GPU (other host threads, other
 *    streams) race; serialise them.  The call synchronises `stream` (a cudaStream_t, NULL = default).
 *  - Returns LBM_ERR_DIVERGED when a population is NaN or Inf (out is still filled).              */
#define LBM_NOALLOC_MAX_CELLS 67108864LL
int  lbm_sums_fp64_noalloc(const void* populations, int lattice, int storage, int64_t nx, int64_t ny,
                           int64_t nz, double storage_scale, void* stream, double out[4]);

/* ---- batched ensemble -------------------------------------------------------------------
 * Many independent lattices (any mix of D2Q9/D3Q27 BGK, sizes and rates, one storage type) advanced
 * together: every step is one persistent kernel launch over a work table that holds the row groups of
 * all members of both families (staged by bulk copies; members with nx a multiple of 16 up to 1024),
 * plus, only if some member's rows cannot be copied that way, one tile launch per family for those
 * (one thread per cell).  nsteps of those are captured in a CUDA graph and replayed.  Every member
 * gives the same populations as stepping it alone.                                               */
int  lbm_batch_create(const lbm_desc* descs, int n, lbm_batch** out);
void lbm_batch_destroy(lbm_batch* b);
int  lbm_batch_size(const lbm_batch* b);
int  lbm_batch_step(lbm_batch* b, int64_t nsteps);
/* Wait for the batch's stream; LBM_ERR_TIMEOUT (once; the error word is cleared) if a bounded wait of
 * the row pipeline gave up. */
int  lbm_batch_sync(lbm_batch* b);
int  lbm_batch_get_populations(lbm_batch* b, int k, void* dst, int dtype, int memory);
int  lbm_batch_set_populations(lbm_batch* b, int k, const void* src, int dtype, int memory);
int  lbm_batch_get_macros(lbm_batch* b, int k, void* rho, void* u, int dtype, int memory);
int  lbm_batch_sums_fp64(lbm_batch* b, int k, double out[4]);
int64_t lbm_batch_cells(const lbm_batch* b);
void* lbm_batch_stream(lbm_batch* b);
/* Tile shape chosen by the autotuner (cells per tile along x, tiles launched per step). */
int  lbm_batch_tile_info(const lbm_batch* b, int* tile_x, int64_t* n_tiles);
/* The configuration in use after the first step: kernel launches per step, and the per-direction copy
 * size the autotuner chose for the one-launch row groups (D2Q9, D3Q27; 0 when not in that mode).     */
int  lbm_batch_plan(const lbm_batch* b, int* launches_per_step, int* group_bytes_d2q9, int* group_bytes_d3q27);
/* Work distribution: AUTO (default) times the candidates on the first step; TILES steps every member
 * with the one-thread-per-cell tile kernel; ROWS uses one row-pipeline launch over the eligible members
 * of both families; ROWS_PER_FAMILY one row-pipeline launch per family (kept for comparison).
 * lbm_batch_get_mode reports the choice in use (AUTO before the first step).                     */
enum lbm_batch_mode { LBM_BATCH_AUTO = 0, LBM_BATCH_TILES = 1, LBM_BATCH_ROWS = 2, LBM_BATCH_ROWS_PER_FAMILY = 3 };
int  lbm_batch_set_mode(lbm_batch* b, int mode);
int  lbm_batch_get_mode(const lbm_batch* b);
/* Test hook of the row pipeline's bounded waits (no counterpart in the reference), as
 * lbm_test_stall_next_step: the next lbm_batch_step launches one step on its own in which work item
 * `item` of each row work table is never filled and every wait gives up after `wait_clocks` clocks;
 * lbm_batch_sync then reports LBM_ERR_TIMEOUT once.  Needs a row mode in use (after a first step).  */
int  lbm_batch_test_stall_next_step(lbm_batch* b, int64_t item, int64_t wait_clocks);

/* ---- problem set-up helpers (the reference's loop-invariant state, layer L3) --------------
 * Each fills mask[N] (column-major) and the descriptor's class table so that the per-cell
 * behaviour equals the reference driver's sequence of overwrites.                              */
/* D2Q9 lid-driven cavity: solid x=0, x=nx-1, y=0; lid row y=ny-1, x=1..nx-2 (cpp/d2q9_bgk_lid.cpp:64,90-91,141-146). */
int lbm_setup_cavity2d(lbm_desc* d, uint8_t* mask, double u_lid);
/* D3Q27 lid-driven cavity: fluid x=1..nx-2, y=1..ny-2, z=1..nz-1; lid plane z=nz-1 (cpp/d3q27_bgk_lid.cpp:119-120,179-186). */
int lbm_setup_cavity3d(lbm_desc* d, uint8_t* mask, double u_lid);
/* D2Q9 channel: solid circle (x-ox)^2+(y-oy)^2 <= r^2 and rows y=0, y=ny-1.  config_mode = 0 gives the
 * reference's equilibrium forcing (inlet u_x + rho=1 at x=0, rho=1 at x=nx-1, periodic in x;
 * cpp/d2q9_bgk_channel_packed.cpp:37-39,64-69).  config_mode = 1 gives an equilibrium inlet
 * (rho=1, u=(u_in,0)) and a zero-gradient outlet; config_mode = 2 a Zou-He velocity inlet
 * (u=(u_in,0)) and a Zou-He pressure outlet (rho=1, uy=0).                                       */
int lbm_setup_channel2d(lbm_desc* d, uint8_t* mask, double u_in, double ox, double oy, double r,
                        int config_mode);
/* D3Q27 duct: walls y=0, y=ny-1, z=0, z=nz-1, solid sphere centre (ox,oy,oz) radius r,
 * equilibrium inlet at x=0, zero-gradient outlet at x=nx-1.                                      */
int lbm_setup_duct3d(lbm_desc* d, uint8_t* mask, double u_in, double ox, double oy, double oz,
                     double r);
/* Index-list shim: accept the reference's solid-node list ON = where(BOUND) (linear column-major
 * indices, cpp/d2q9_bgk_lid.cpp:94) and mark those cells with class `cls`.                      */
int lbm_mask_from_index_list(uint8_t* mask, int64_t n_cells, const int64_t* on, int64_t n_on,
                             uint8_t cls);
/* Reference-driver relaxation rules: tau = 3 nu + 1/2, omega = 1/tau with
 *   rule 0: nu = u * L / Re        (C++ drivers, cpp/d2q9_bgk_lid.cpp:45)
 *   rule 1: nu = u * 2 * L / Re    (Rust drivers, rust/examples/d2q9_bgk_lid.rs:52)            */
double lbm_omega_from_re(double u, double L, double re, int rule);
/* MRT rate vector of the reference (s0=s1=1.3, sv=1.1, sb=0.9, ...; rust/examples/d3q27_mrt_lid.rs:111-150). */
void lbm_mrt_reference_rates(double s[27]);
/* MRT rates with shear rate sv for rows 4-6,8,9 and `other` for every other row. */
void lbm_mrt_rates(double s[27], double sv, double other);
/* One host-side MRT collision of a single cell (FP64): f_out = M^-1 (m - S (m - meq(rho,u))), m = M f_in.
 * Used for the reference's MRT start state (rust/examples/d3q27_mrt_lid.rs:228-287).             */
int lbm_mrt_collide_host(const lbm_desc* d, const double f_in[27], double rho, const double u[3],
                         double f_out[27]);

#ifdef __cplusplus
}
#endif
#endif /* LBM_B200_H */
