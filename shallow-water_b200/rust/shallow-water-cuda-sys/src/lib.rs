//! Raw bindings of libswcuda.so: every entry point of include/sw_cuda.h, the
//! status codes, the precisions and the field indices of nhswps::State
//! (src/nhswps/mod.rs:87-148 of the reference).  All arrays are float64 in the
//! reference's Fortran order unless an entry point says otherwise.  The safe
//! wrappers are in the shallow-water-cuda crate.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_double, c_float, c_int, c_longlong, c_void};

/// The opaque context (sw_ctx): one ensemble of members of one (ng, nz) on one device.
#[repr(C)]
pub struct SwCtx {
    _private: [u8; 0],
}

/// The opaque ensemble of members with uneven grids (sw_ensemble).
#[repr(C)]
pub struct SwEnsemble {
    _private: [u8; 0],
}

pub const SW_OK: c_int = 0;
pub const SW_ERR_FACTORISE: c_int = 1;
pub const SW_ERR_CUDA: c_int = 2;
pub const SW_ERR_PSOLVE_DIVERGED: c_int = 3;
pub const SW_ERR_PSOLVE_MAXITER: c_int = 4;
pub const SW_ERR_ARG: c_int = 6;
pub const SW_ERR_STATE: c_int = 7;

pub const SW_FP64: c_int = 0;
pub const SW_MIXED: c_int = 1;
pub const SW_FP32: c_int = 2;

pub const SW_U: c_int = 0;
pub const SW_V: c_int = 1;
pub const SW_W: c_int = 2;
pub const SW_Z: c_int = 3;
pub const SW_ZX: c_int = 4;
pub const SW_ZY: c_int = 5;
pub const SW_R: c_int = 6;
pub const SW_RI: c_int = 7;
pub const SW_AA: c_int = 8;
pub const SW_ZETA: c_int = 9;
pub const SW_PN: c_int = 10;
pub const SW_DPN: c_int = 11;
pub const SW_PS: c_int = 12;
pub const SW_QS: c_int = 13;
pub const SW_DS: c_int = 14;
pub const SW_GS: c_int = 15;
pub const SW_NFIELDS: c_int = 16;

#[link(name = "swcuda")]
extern "C" {
pub fn sw_last_error() -> *const c_char;
    pub fn sw_version() -> c_int;
    pub fn sw_factorisen(n: c_int, factors: *mut c_int) -> c_int;
    pub fn sw_initfft(n: c_int, factors: *mut c_int, trig: *mut c_double) -> c_int;
    pub fn sw_forfft(m: c_int, n: c_int, x: *mut c_double, trig: *const c_double, factors: *const c_int) -> c_int;
    pub fn sw_revfft(m: c_int, n: c_int, x: *mut c_double, trig: *const c_double, factors: *const c_int) -> c_int;
    pub fn sw_forfft_dev(m: c_int, n: c_int, x: *mut c_void, precision: c_int, stream: *mut c_void) -> c_int;
    pub fn sw_revfft_dev(m: c_int, n: c_int, x: *mut c_void, precision: c_int, stream: *mut c_void) -> c_int;
    pub fn sw_ctx_create(ng: c_int, nz: c_int, nmembers: c_int, precision: c_int, device: c_int, out: *mut *mut SwCtx) -> c_int;
    pub fn sw_ctx_destroy(ctx: *mut SwCtx);
    pub fn sw_ctx_info(ctx: *const SwCtx, ng: *mut c_int, nz: *mut c_int, nmembers: *mut c_int, precision: *mut c_int) -> c_int;
    pub fn sw_spectral_get(ctx: *mut SwCtx, name: *const c_char, out: *mut c_double, n: usize) -> c_int;
    pub fn sw_state_set(ctx: *mut SwCtx, field: c_int, member: c_int, host: *const c_double, n: usize) -> c_int;
    pub fn sw_state_get(ctx: *mut SwCtx, field: c_int, member: c_int, host: *mut c_double, n: usize) -> c_int;
    pub fn sw_state_set_all(ctx: *mut SwCtx, field: c_int, host: *const c_double, n: usize) -> c_int;
    pub fn sw_state_get_all(ctx: *mut SwCtx, field: c_int, host: *mut c_double, n: usize) -> c_int;
    pub fn sw_state_set_all_async(ctx: *mut SwCtx, field: c_int, host: *const c_double, n: usize) -> c_int;
    pub fn sw_state_get_all_async(ctx: *mut SwCtx, field: c_int, host: *mut c_double, n: usize) -> c_int;
    pub fn sw_set_time(ctx: *mut SwCtx, t: c_double) -> c_int;
    pub fn sw_get_time(ctx: *const SwCtx, t: *mut c_double) -> c_int;
    pub fn sw_ptospc(ctx: *mut SwCtx, rvar: *const c_double, svar: *mut c_double) -> c_int;
    pub fn sw_spctop(ctx: *mut SwCtx, svar: *const c_double, rvar: *mut c_double) -> c_int;
    pub fn sw_xderiv(ctx: *mut SwCtx, var: *const c_double, der: *mut c_double) -> c_int;
    pub fn sw_yderiv(ctx: *mut SwCtx, var: *const c_double, der: *mut c_double) -> c_int;
    pub fn sw_jacob(ctx: *mut SwCtx, aa: *const c_double, bb: *const c_double, cs: *mut c_double) -> c_int;
    pub fn sw_divs(ctx: *mut SwCtx, aa: *const c_double, bb: *const c_double, cs: *mut c_double) -> c_int;
    pub fn sw_deal2d(ctx: *mut SwCtx, fp: *mut c_double) -> c_int;
    pub fn sw_deal3d(ctx: *mut SwCtx, fp: *mut c_double) -> c_int;
    pub fn sw_ptospc3d(ctx: *mut SwCtx, fp: *const c_double, fs: *mut c_double, izbeg: c_int, izend: c_int) -> c_int;
    pub fn sw_spctop3d(ctx: *mut SwCtx, fs: *const c_double, fp: *mut c_double, izbeg: c_int, izend: c_int) -> c_int;
    pub fn sw_spec1d(ctx: *mut SwCtx, ss: *const c_double, spec: *mut c_double) -> c_int;
    pub fn sw_balinit(ctx: *mut SwCtx, qq_init: *const c_double, qq: *mut c_double, dd: *mut c_double, gg: *mut c_double, iters: *mut c_int) -> c_int;
    pub fn sw_main_invert(ctx: *mut SwCtx) -> c_int;
    pub fn sw_vertical(ctx: *mut SwCtx) -> c_int;
    pub fn sw_coeffs(ctx: *mut SwCtx, sigx: *mut c_double, sigy: *mut c_double, cpt1: *mut c_double, cpt2: *mut c_double) -> c_int;
    pub fn sw_cpsource(ctx: *mut SwCtx, sp0: *mut c_double) -> c_int;
    pub fn sw_psolve(ctx: *mut SwCtx, nitmax: c_int, iters: *mut c_int, errp: *mut c_double) -> c_int;
    pub fn sw_source(ctx: *mut SwCtx, sqs: *mut c_double, sds: *mut c_double, sgs: *mut c_double) -> c_int;
    pub fn sw_advance(ctx: *mut SwCtx, nsteps: c_int, ggen: c_int) -> c_int;
    pub fn sw_set_graphs(ctx: *mut SwCtx, enable: c_int) -> c_int;
    pub fn sw_set_psolve_toler(ctx: *mut SwCtx, toler: c_double) -> c_int;
    pub fn sw_set_psolve_relax(ctx: *mut SwCtx, omega: c_double) -> c_int;
    pub fn sw_sweep_counts(ctx: *mut SwCtx, out: *mut c_longlong) -> c_int;
    pub fn sw_set_fft_chunk(ctx: *mut SwCtx, planes: c_int, in_use: *mut c_int) -> c_int;
    pub fn sw_set_fft_single_pass(ctx: *mut SwCtx, enable: c_int, in_use: *mut c_int) -> c_int;
    pub fn sw_set_fft_overlap(ctx: *mut SwCtx, enable: c_int, in_use: *mut c_int) -> c_int;
    pub fn sw_set_fft_tile(ctx: *mut SwCtx, columns: c_int, in_use: *mut c_int) -> c_int;
    pub fn sw_autotune_fft(ctx: *mut SwCtx, reps: c_int, maxc: c_int, tiles: *mut c_int, chunks: *mut c_int, overlaps: *mut c_int, ms: *mut c_float, ncand: *mut c_int, chosen_tile: *mut c_int, chosen_chunk: *mut c_int, chosen_overlap: *mut c_int) -> c_int;
    pub fn sw_diagnose(ctx: *mut SwCtx, member: c_int, out: *mut c_double) -> c_int;
    pub fn sw_diag_history(ctx: *mut SwCtx, out: *mut c_double, cap: c_int, count: *mut c_int) -> c_int;
    pub fn sw_energy(ctx: *mut SwCtx, member: c_int, out: *mut c_double) -> c_int;
    pub fn sw_savegrid(ctx: *mut SwCtx, member: c_int, energies: *mut c_double, spectra: *mut c_double, nspec: c_int, fields3: *mut c_float, fields2: *mut c_float) -> c_int;
    pub fn sw_last_sweeps(ctx: *mut SwCtx, out: *mut c_int) -> c_int;
    pub fn sw_advance_async(ctx: *mut SwCtx, nsteps: c_int, ggen: c_int) -> c_int;
    pub fn sw_sync(ctx: *mut SwCtx) -> c_int;
    pub fn sw_field_device_ptr(ctx: *mut SwCtx, field: c_int, ptr: *mut *mut c_void, elem_bytes: *mut c_int) -> c_int;
    pub fn sw_tridiag_batched(n: c_int, nsys: c_int, a: *const c_double, b: *const c_double, c: *const c_double, d: *const c_double, x: *mut c_double, stream: *mut c_void) -> c_int;
    pub fn sw_tridiag_batched_host(n: c_int, nsys: c_int, a: *const c_double, b: *const c_double, c: *const c_double, d: *const c_double, x: *mut c_double) -> c_int;
    pub fn sw_stream(ctx: *mut SwCtx, stream: *mut *mut c_void) -> c_int;
    pub fn sw_fft2d_dev(ctx: *mut SwCtx, direction: c_int, nplanes: c_int, in_: *const c_void, out: *mut c_void) -> c_int;
    pub fn sw_fft2d_noalloc(ng: c_int, direction: c_int, nplanes: c_int, in_: *const c_double, out: *mut c_double, stream: *mut c_void) -> c_int;
    pub fn sw_ensemble_create(ng: *const c_int, nz: *const c_int, nmembers: c_int, precision: c_int, device: c_int, out: *mut *mut SwEnsemble) -> c_int;
    pub fn sw_ensemble_destroy(e: *mut SwEnsemble);
    pub fn sw_ensemble_info(e: *const SwEnsemble, nmembers: *mut c_int, ngroups: *mut c_int) -> c_int;
    pub fn sw_ensemble_stream(e: *mut SwEnsemble, stream: *mut *mut c_void) -> c_int;
    pub fn sw_ensemble_member(e: *mut SwEnsemble, member: c_int, ctx: *mut *mut SwCtx, index: *mut c_int) -> c_int;
    pub fn sw_ensemble_advance(e: *mut SwEnsemble, nsteps: c_int, ggen: c_int) -> c_int;
    pub fn sw_ensemble_advance_async(e: *mut SwEnsemble, nsteps: c_int, ggen: c_int) -> c_int;
    pub fn sw_ensemble_sync(e: *mut SwEnsemble) -> c_int;
    pub fn sw_kernel_launches(ctx: *mut SwCtx, count: *mut c_longlong) -> c_int;
}
