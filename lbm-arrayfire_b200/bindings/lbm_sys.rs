//! lbm_sys.rs — Rust declarations of the liblbm_b200 C ABI (include/lbm.h), for the reference's Rust
//! examples (rust/examples/d2q9_bgk_lid.rs, d2q9_bgk_channel.rs, d3q27_bgk_lid.rs, d3q27_mrt_lid.rs,
//! d3q27_mrt_channel.rs) to call instead of their ArrayFire time loops.  Drop the file into the crate
//! (`mod lbm_sys;`) and link the library from build.rs:
//!
//! ```text
//! println!("cargo:rustc-link-search=native=<repo>/lbm-arrayfire_b200/lbm_b200");
//! println!("cargo:rustc-link-lib=dylib=lbm_b200");
//! ```
//!
//! The structs are `#[repr(C)]` mirrors of lbm_cell_class and lbm_desc; the const assertions at the
//! end pin their sizes and field offsets, which tests/test_bindings.py checks against the C layout that
//! gcc gives the header (bindings/c_abi_check.c).  Every function is `unsafe` (raw pointers across the
//! boundary) and returns the header's status codes; lbm_last_error() gives the message.
#![allow(non_camel_case_types, non_snake_case, dead_code)]

use std::os::raw::{c_char, c_double, c_float, c_int, c_void};

pub const LBM_ABI_VERSION: c_int = 1;

pub const LBM_OK: c_int = 0;
pub const LBM_ERR_INVALID: c_int = -1;
pub const LBM_ERR_CUDA: c_int = -2;
pub const LBM_ERR_NOMEM: c_int = -3;
pub const LBM_ERR_DIVERGED: c_int = -4;
pub const LBM_ERR_UNSUPPORTED: c_int = -5;
pub const LBM_ERR_NO_DEVICE: c_int = -6;
pub const LBM_ERR_STATE: c_int = -7;
pub const LBM_ERR_TIMEOUT: c_int = -8;

pub const LBM_D2Q9: c_int = 0;
pub const LBM_D3Q27: c_int = 1;
pub const LBM_BGK: c_int = 0;
pub const LBM_MRT: c_int = 1;
pub const LBM_SHANCHEN: c_int = 2;
pub const LBM_F32: c_int = 0;
pub const LBM_F16S: c_int = 1;
pub const LBM_BF16S: c_int = 2;
pub const LBM_F64: c_int = 3;
pub const LBM_MRT_REF: c_int = 0;
pub const LBM_MRT_GRAM_SCHMIDT: c_int = 1;
pub const LBM_ARITH_DEVIATION: c_int = 0;
pub const LBM_ARITH_ABSOLUTE: c_int = 1;
pub const LBM_ROUND_STOCHASTIC: c_int = 0;
pub const LBM_ROUND_NEAREST: c_int = 1;
pub const LBM_DTYPE_F32: c_int = 0;
pub const LBM_DTYPE_F64: c_int = 1;
pub const LBM_HOST: c_int = 0;
pub const LBM_DEVICE: c_int = 1;
pub const LBM_KERNEL_AUTO: c_int = 0;
pub const LBM_KERNEL_PLAIN: c_int = 1;
pub const LBM_KERNEL_ROWS: c_int = 2;
pub const LBM_KERNEL_CLUSTER: c_int = 3;
pub const LBM_BATCH_AUTO: c_int = 0;
pub const LBM_BATCH_TILES: c_int = 1;
pub const LBM_BATCH_ROWS: c_int = 2;
pub const LBM_BATCH_ROWS_PER_FAMILY: c_int = 3;

pub const LBM_MAX_CLASSES: usize = 16;
pub const LBM_CELL_BOUNCE: u32 = 0x01;
pub const LBM_CELL_SET_RHO: u32 = 0x02;
pub const LBM_CELL_SET_UX: u32 = 0x04;
pub const LBM_CELL_SET_UY: u32 = 0x08;
pub const LBM_CELL_SET_UZ: u32 = 0x10;
pub const LBM_CELL_EQUILIBRIUM: u32 = 0x20;
pub const LBM_CELL_ZEROGRAD_XP: u32 = 0x40;
pub const LBM_CELL_ZOUHE_VEL_XM: u32 = 0x80;
pub const LBM_CELL_ZOUHE_RHO_XP: u32 = 0x100;
pub const LBM_NOALLOC_MAX_CELLS: i64 = 67108864;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct lbm_cell_class {
    pub flags: u32,
    pub reserved: u32,
    pub rho: c_double,
    pub ux: c_double,
    pub uy: c_double,
    pub uz: c_double,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct lbm_desc {
    pub lattice: i32,
    pub collision: i32,
    pub storage: i32,
    pub mrt_basis: i32,
    pub arithmetic: i32,
    pub rounding: i32,
    pub nx: i64,
    pub ny: i64,
    pub nz: i64,
    pub omega: c_double,
    pub mrt_s: [c_double; 27],
    pub sc_G: c_double,
    pub storage_scale: c_double,
    pub n_classes: i32,
    pub device: i32,
    pub classes: [lbm_cell_class; LBM_MAX_CLASSES],
    pub mask: *const u8,
}

/// Opaque single-lattice context.
#[repr(C)]
pub struct lbm_ctx {
    _opaque: [u8; 0],
}

/// Opaque ensemble.
#[repr(C)]
pub struct lbm_batch {
    _opaque: [u8; 0],
}

extern "C" {
    pub fn lbm_abi_version() -> c_int;
    pub fn lbm_strerror(status: c_int) -> *const c_char;
    pub fn lbm_last_error() -> *const c_char;
    pub fn lbm_desc_init(d: *mut lbm_desc, lattice: c_int, collision: c_int, storage: c_int, nx: i64, ny: i64, nz: i64);
    pub fn lbm_q(lattice: c_int) -> c_int;
    pub fn lbm_velocities(lattice: c_int, cx: *mut i32, cy: *mut i32, cz: *mut i32, w: *mut c_double, opp: *mut i32) -> c_int;

    pub fn lbm_create(d: *const lbm_desc, out: *mut *mut lbm_ctx) -> c_int;
    pub fn lbm_destroy(c: *mut lbm_ctx);
    pub fn lbm_set_populations(c: *mut lbm_ctx, src: *const c_void, dtype: c_int, memory: c_int) -> c_int;
    pub fn lbm_get_populations(c: *mut lbm_ctx, dst: *mut c_void, dtype: c_int, memory: c_int) -> c_int;
    pub fn lbm_init_equilibrium(c: *mut lbm_ctx, rho: *const c_double, u: *const c_double) -> c_int;
    pub fn lbm_step(c: *mut lbm_ctx, nsteps: i64) -> c_int;
    pub fn lbm_sync(c: *mut lbm_ctx) -> c_int;
    pub fn lbm_get_macros(c: *mut lbm_ctx, rho: *mut c_void, u: *mut c_void, dtype: c_int, memory: c_int) -> c_int;
    pub fn lbm_sums_fp64(c: *mut lbm_ctx, out: *mut c_double) -> c_int;
    pub fn lbm_residual_fp64(c: *mut lbm_ctx, out: *mut c_double) -> c_int;
    pub fn lbm_last_step_ms(c: *mut lbm_ctx, ms: *mut c_float) -> c_int;
    pub fn lbm_steps_done(c: *const lbm_ctx) -> i64;
    pub fn lbm_stream(c: *mut lbm_ctx) -> *mut c_void;
    pub fn lbm_set_stream(c: *mut lbm_ctx, stream: *mut c_void) -> c_int;
    pub fn lbm_device_populations(c: *mut lbm_ctx, bytes: *mut usize) -> *mut c_void;
    pub fn lbm_get_desc(c: *const lbm_ctx, out: *mut lbm_desc) -> c_int;
    pub fn lbm_face_get(c: *mut lbm_ctx, plane: i64, dirs: *const i32, ndirs: i32, dst: *mut c_void, memory: c_int) -> c_int;
    pub fn lbm_face_set(c: *mut lbm_ctx, plane: i64, dirs: *const i32, ndirs: i32, src: *const c_void, memory: c_int) -> c_int;
    pub fn lbm_step_planes(c: *mut lbm_ctx, first: i64, count: i64, stride: i64, finish: c_int,
                           stream: *mut c_void) -> c_int;
    pub fn lbm_set_reserved_sms(c: *mut lbm_ctx, sms: c_int) -> c_int;
    pub fn lbm_device_buffers(c: *mut lbm_ctx, current: *mut *mut c_void, next: *mut *mut c_void,
                              bytes: *mut usize) -> c_int;
    pub fn lbm_set_cell_offset(c: *mut lbm_ctx, offset: i64) -> c_int;
    pub fn lbm_set_block(c: *mut lbm_ctx, threads_x: c_int) -> c_int;
    pub fn lbm_get_block(c: *const lbm_ctx) -> c_int;
    pub fn lbm_set_kernel(c: *mut lbm_ctx, kind: c_int) -> c_int;
    pub fn lbm_get_kernel(c: *const lbm_ctx) -> c_int;
    pub fn lbm_test_stall_next_step(c: *mut lbm_ctx, item: i64, wait_clocks: i64) -> c_int;
    pub fn lbm_test_index64(c: *mut lbm_ctx, on: c_int) -> c_int;

    pub fn lbm_sums_fp64_noalloc(populations: *const c_void, lattice: c_int, storage: c_int, nx: i64, ny: i64, nz: i64,
                                 storage_scale: c_double, stream: *mut c_void, out: *mut c_double) -> c_int;

    pub fn lbm_batch_create(descs: *const lbm_desc, n: c_int, out: *mut *mut lbm_batch) -> c_int;
    pub fn lbm_batch_destroy(b: *mut lbm_batch);
    pub fn lbm_batch_size(b: *const lbm_batch) -> c_int;
    pub fn lbm_batch_step(b: *mut lbm_batch, nsteps: i64) -> c_int;
    pub fn lbm_batch_sync(b: *mut lbm_batch) -> c_int;
    pub fn lbm_batch_get_populations(b: *mut lbm_batch, k: c_int, dst: *mut c_void, dtype: c_int, memory: c_int) -> c_int;
    pub fn lbm_batch_set_populations(b: *mut lbm_batch, k: c_int, src: *const c_void, dtype: c_int, memory: c_int) -> c_int;
    pub fn lbm_batch_get_macros(b: *mut lbm_batch, k: c_int, rho: *mut c_void, u: *mut c_void, dtype: c_int, memory: c_int) -> c_int;
    pub fn lbm_batch_sums_fp64(b: *mut lbm_batch, k: c_int, out: *mut c_double) -> c_int;
    pub fn lbm_batch_cells(b: *const lbm_batch) -> i64;
    pub fn lbm_batch_stream(b: *mut lbm_batch) -> *mut c_void;
    pub fn lbm_batch_tile_info(b: *const lbm_batch, tile_x: *mut c_int, n_tiles: *mut i64) -> c_int;
    pub fn lbm_batch_plan(b: *const lbm_batch, launches_per_step: *mut c_int, group_bytes_d2q9: *mut c_int,
                          group_bytes_d3q27: *mut c_int) -> c_int;
    pub fn lbm_batch_set_mode(b: *mut lbm_batch, mode: c_int) -> c_int;
    pub fn lbm_batch_get_mode(b: *const lbm_batch) -> c_int;
    pub fn lbm_batch_test_stall_next_step(b: *mut lbm_batch, item: i64, wait_clocks: i64) -> c_int;

    pub fn lbm_setup_cavity2d(d: *mut lbm_desc, mask: *mut u8, u_lid: c_double) -> c_int;
    pub fn lbm_setup_cavity3d(d: *mut lbm_desc, mask: *mut u8, u_lid: c_double) -> c_int;
    pub fn lbm_setup_channel2d(d: *mut lbm_desc, mask: *mut u8, u_in: c_double, ox: c_double, oy: c_double, r: c_double,
                               config_mode: c_int) -> c_int;
    pub fn lbm_setup_duct3d(d: *mut lbm_desc, mask: *mut u8, u_in: c_double, ox: c_double, oy: c_double, oz: c_double,
                            r: c_double) -> c_int;
    pub fn lbm_mask_from_index_list(mask: *mut u8, n_cells: i64, on: *const i64, n_on: i64, cls: u8) -> c_int;
    pub fn lbm_omega_from_re(u: c_double, L: c_double, re: c_double, rule: c_int) -> c_double;
    pub fn lbm_mrt_reference_rates(s: *mut c_double);
    pub fn lbm_mrt_rates(s: *mut c_double, sv: c_double, other: c_double);
    pub fn lbm_mrt_collide_host(d: *const lbm_desc, f_in: *const c_double, rho: c_double, u: *const c_double,
                                f_out: *mut c_double) -> c_int;
}

// Layout of the mirrored structs on LP64 targets (x86-64, aarch64): the same numbers that gcc gives
// include/lbm.h (checked by tests/test_bindings.py through bindings/c_abi_check.c).
const _: () = assert!(std::mem::size_of::<lbm_cell_class>() == 40);
const _: () = assert!(std::mem::offset_of!(lbm_cell_class, flags) == 0);
const _: () = assert!(std::mem::offset_of!(lbm_cell_class, reserved) == 4);
const _: () = assert!(std::mem::offset_of!(lbm_cell_class, rho) == 8);
const _: () = assert!(std::mem::offset_of!(lbm_cell_class, ux) == 16);
const _: () = assert!(std::mem::offset_of!(lbm_cell_class, uy) == 24);
const _: () = assert!(std::mem::offset_of!(lbm_cell_class, uz) == 32);
const _: () = assert!(std::mem::size_of::<lbm_desc>() == 944);
const _: () = assert!(std::mem::offset_of!(lbm_desc, lattice) == 0);
const _: () = assert!(std::mem::offset_of!(lbm_desc, collision) == 4);
const _: () = assert!(std::mem::offset_of!(lbm_desc, storage) == 8);
const _: () = assert!(std::mem::offset_of!(lbm_desc, mrt_basis) == 12);
const _: () = assert!(std::mem::offset_of!(lbm_desc, arithmetic) == 16);
const _: () = assert!(std::mem::offset_of!(lbm_desc, rounding) == 20);
const _: () = assert!(std::mem::offset_of!(lbm_desc, nx) == 24);
const _: () = assert!(std::mem::offset_of!(lbm_desc, ny) == 32);
const _: () = assert!(std::mem::offset_of!(lbm_desc, nz) == 40);
const _: () = assert!(std::mem::offset_of!(lbm_desc, omega) == 48);
const _: () = assert!(std::mem::offset_of!(lbm_desc, mrt_s) == 56);
const _: () = assert!(std::mem::offset_of!(lbm_desc, sc_G) == 272);
const _: () = assert!(std::mem::offset_of!(lbm_desc, storage_scale) == 280);
const _: () = assert!(std::mem::offset_of!(lbm_desc, n_classes) == 288);
const _: () = assert!(std::mem::offset_of!(lbm_desc, device) == 292);
const _: () = assert!(std::mem::offset_of!(lbm_desc, classes) == 296);
const _: () = assert!(std::mem::offset_of!(lbm_desc, mask) == 936);

/// The loop of rust/examples/d2q9_bgk_lid.rs:151-236 on the library: set up the cavity, step
/// `iterations` times, return the FP64 mass and momentum sums (a sketch of how an example calls it).
pub unsafe fn d2q9_lid_cavity(nx: i64, ny: i64, u_lid: f64, re: f64, iterations: i64) -> Result<[f64; 4], c_int> {
    let mut d: lbm_desc = std::mem::zeroed();
    lbm_desc_init(&mut d, LBM_D2Q9, LBM_BGK, LBM_F32, nx, ny, 1);
    d.omega = lbm_omega_from_re(u_lid, nx as f64, re, 1); // the Rust examples' viscosity rule (:52)
    let mut mask = vec![0u8; (nx * ny) as usize];
    let rc = lbm_setup_cavity2d(&mut d, mask.as_mut_ptr(), u_lid);
    if rc != LBM_OK { return Err(rc); }
    let mut ctx: *mut lbm_ctx = std::ptr::null_mut();
    let rc = lbm_create(&d, &mut ctx);
    if rc != LBM_OK { return Err(rc); }
    let mut out = [0.0f64; 4];
    let mut rc = lbm_step(ctx, iterations);
    if rc == LBM_OK { rc = lbm_sync(ctx); }
    if rc == LBM_OK { rc = lbm_sums_fp64(ctx, out.as_mut_ptr()); }
    lbm_destroy(ctx);
    if rc != LBM_OK { Err(rc) } else { Ok(out) }
}
