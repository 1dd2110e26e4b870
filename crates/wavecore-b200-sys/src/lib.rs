//! Raw bindings to `include/wavecore_c.h`, the C ABI of the B200 implementation of wavecore's time
//! step (`wavecore::Solver::step`, crates/wavecore/src/solver.rs:479-507 of mlaegn/wavesim).
//!
//! Every item mirrors the header one for one: the same names, the same field order and the same
//! argument order, so that `wavecore` can put a `B200Solver` behind a cargo feature and call
//! these where it calls `Solver` today. The safe wrapper is not part of this crate.
#![allow(non_camel_case_types)]
#![no_std]

use core::ffi::{c_char, c_void};

/// Ghost layers on every side of a padded array (crates/wavecore/src/grid.rs:4).
pub const WC_GHOST: usize = 3;
/// Kinds of kernel that `wc_profile_read` reports.
pub const WC_KERNEL_KINDS: usize = 5;

pub type wc_status = i32;
pub const WC_OK: wc_status = 0;
pub const WC_EINVAL: wc_status = 1;
pub const WC_EPERIODIC: wc_status = 2;
pub const WC_ENAN: wc_status = 3;
pub const WC_EUNCONVERGED: wc_status = 4;
pub const WC_ETIMEOUT: wc_status = 5;
pub const WC_ECUDA: wc_status = 6;
pub const WC_ENOMEM: wc_status = 7;
pub const WC_EUNSUPPORTED: wc_status = 8;

pub type wc_order = i32;
pub const WC_ORDER_FIRST: wc_order = 0;
pub const WC_ORDER_SECOND: wc_order = 1;
pub const WC_ORDER_FIFTH: wc_order = 2;

pub type wc_preconditioner = i32;
pub const WC_PC_JACOBI: wc_preconditioner = 0;
pub const WC_PC_LEARNED: wc_preconditioner = 1;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_grid {
    pub nx: u64,
    pub ny: u64,
    pub dx: f64,
    pub dy: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_sponge {
    pub width: u64,
    pub strength: f64,
    pub level: f64,
    pub west: i32,
    pub east: i32,
    pub south: i32,
    pub north: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_wavemaker {
    pub x: f64,
    pub amplitude: f64,
    pub period: f64,
    pub angle: f64,
    pub sigma: f64,
    pub ramp_periods: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_eddy {
    pub initial: f64,
    pub settled: f64,
    pub duration: f64,
    pub mixing: f64,
    pub linger: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_breaking {
    pub eta_ratio_lo: f64,
    pub eta_ratio_hi: f64,
    pub slope_lo: f64,
    pub slope_hi: f64,
    pub viscosity: i32,
    pub eddy: wc_eddy,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_dispersion {
    pub breaking: wc_breaking,
    pub nonlinear: i32,
    pub tolerance: f64,
    pub max_iterations: u64,
    pub preconditioner: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct wc_config {
    pub cfl: f64,
    pub order: i32,
    pub manning: f64,
    pub periodic_y: i32,
    pub sponges: *const wc_sponge,
    pub n_sponges: u64,
    pub wavemaker: *const wc_wavemaker,
    pub dispersion: *const wc_dispersion,
    pub shallow_cells: *const u8,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_stats {
    pub solves: u64,
    pub iterations: u64,
    pub unconverged: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_limiting {
    pub i: u64,
    pub j: u64,
    pub depth: f64,
    pub speed: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_diagnostics {
    pub volume: f64,
    pub max_abs_momentum: f64,
    pub min_depth: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_kernel_time {
    pub launches: u64,
    pub total_ms: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct wc_record_summary {
    pub seconds: f64,
    pub waves: u64,
    pub has_harmonic: i32,
    pub has_unsettled: i32,
    pub unsettled: f64,
}

/// Opaque handles.
#[repr(C)]
pub struct wc_solver {
    _private: [u8; 0],
}
#[repr(C)]
pub struct wc_ensemble {
    _private: [u8; 0],
}
#[repr(C)]
pub struct wc_lpc {
    _private: [u8; 0],
}
#[repr(C)]
pub struct wc_recorder {
    _private: [u8; 0],
}
#[repr(C)]
pub struct wc_nest {
    _private: [u8; 0],
}

extern "C" {
    // Defaults of the reference's builders.
    pub fn wc_config_default(cfg: *mut wc_config);
    pub fn wc_dispersion_default(d: *mut wc_dispersion);
    pub fn wc_eddy_default(e: *mut wc_eddy);

    // `Solver` (crates/wavecore/src/solver.rs).
    pub fn wc_solver_create(grid: *const wc_grid, bed_padded: *const f64, cfg: *const wc_config,
                            out: *mut *mut wc_solver) -> wc_status;
    pub fn wc_solver_destroy(s: *mut wc_solver);
    pub fn wc_step(s: *mut wc_solver, h: *mut f64, hu: *mut f64, hv: *mut f64, breaking: *mut f64,
                   time: *mut f64, dt: f64) -> wc_status;
    pub fn wc_stable_dt(s: *mut wc_solver, h: *const f64, hu: *const f64, hv: *const f64,
                        dt_out: *mut f64) -> wc_status;
    pub fn wc_limiting_cell(s: *mut wc_solver, h: *const f64, hu: *const f64, hv: *const f64,
                            out: *mut wc_limiting, found: *mut i32) -> wc_status;
    pub fn wc_breaking_indicator(s: *mut wc_solver, h: *const f64, hu: *const f64, hv: *const f64,
                                 breaking: *const f64, out_interior: *mut f64) -> wc_status;
    pub fn wc_follow_breaking(s: *mut wc_solver, h: *mut f64, hu: *mut f64, hv: *mut f64,
                              breaking: *mut f64, dt: f64, sub_steps: *mut i32) -> wc_status;
    pub fn wc_dispersion_stats(s: *mut wc_solver, out: *mut wc_stats, has: *mut i32) -> wc_status;

    // The device-resident throughput path.
    pub fn wc_state_upload(s: *mut wc_solver, h: *const f64, hu: *const f64, hv: *const f64,
                           time: f64) -> wc_status;
    pub fn wc_breaking_upload(s: *mut wc_solver, breaking: *const f64) -> wc_status;
    pub fn wc_breaking_download(s: *mut wc_solver, breaking: *mut f64) -> wc_status;
    pub fn wc_state_download(s: *mut wc_solver, h: *mut f64, hu: *mut f64, hv: *mut f64,
                             time: *mut f64) -> wc_status;
    pub fn wc_step_device(s: *mut wc_solver, dt: f64) -> wc_status;
    pub fn wc_step_n(s: *mut wc_solver, n_steps: u64, t_end: f64) -> wc_status;
    pub fn wc_stable_dt_device(s: *mut wc_solver, dt_out: *mut f64) -> wc_status;
    pub fn wc_diagnostics_device(s: *mut wc_solver, out: *mut wc_diagnostics) -> wc_status;
    pub fn wc_dispersion_system(s: *mut wc_solver, c: *mut f64, heff: *mut f64, bx: *mut f64,
                                by: *mut f64, wx: *mut f64, wy: *mut f64) -> wc_status;
    pub fn wc_time_device(s: *mut wc_solver, time_out: *mut f64) -> wc_status;
    pub fn wc_set_wait_limit(s: *mut wc_solver, ns: u64) -> wc_status;
    pub fn wc_synchronize(s: *mut wc_solver) -> wc_status;
    pub fn wc_set_stream(s: *mut wc_solver, stream: *mut c_void) -> wc_status;
    pub fn wc_profile_enable(s: *mut wc_solver, on: i32) -> wc_status;
    pub fn wc_profile_read(s: *mut wc_solver, out: *mut wc_kernel_time) -> wc_status;

    // The time-step limit on caller-owned device arrays, allocating nothing.
    pub fn wc_stable_dt_noalloc(grid: *const wc_grid, cfl: f64, d_h: *const f64, d_hu: *const f64,
                                d_hv: *const f64, stream: *mut c_void, dt_out: *mut f64) -> wc_status;

    // Ensembles of independent runs.
    pub fn wc_ensemble_create(n: u64, grids: *const wc_grid, beds: *const *const f64,
                              cfgs: *const wc_config, out: *mut *mut wc_ensemble) -> wc_status;
    pub fn wc_ensemble_destroy(e: *mut wc_ensemble);
    pub fn wc_ensemble_upload(e: *mut wc_ensemble, member: u64, h: *const f64, hu: *const f64,
                              hv: *const f64, time: f64) -> wc_status;
    pub fn wc_ensemble_download(e: *mut wc_ensemble, member: u64, h: *mut f64, hu: *mut f64,
                                hv: *mut f64, time: *mut f64) -> wc_status;
    pub fn wc_ensemble_step_n(e: *mut wc_ensemble, n_steps: u64, t_end: f64) -> wc_status;
    pub fn wc_ensemble_autotune(e: *mut wc_ensemble, trial_steps: u32, choice: *mut i32,
                                ms_per_step: *mut f64) -> wc_status;
    pub fn wc_ensemble_set_lpc(e: *mut wc_ensemble, l: *mut wc_lpc) -> wc_status;
    pub fn wc_ensemble_synchronize(e: *mut wc_ensemble) -> wc_status;
    pub fn wc_ensemble_member_stats(e: *mut wc_ensemble, member: u64, stats: *mut wc_stats,
                                    time: *mut f64) -> wc_status;
    pub fn wc_ensemble_launch_count(e: *const wc_ensemble) -> u64;

    // The learned preconditioner.
    pub fn wc_lpc_create(channels: *const i32, gate_hidden: i32, stride: i32, seed: u64,
                         out: *mut *mut wc_lpc) -> wc_status;
    pub fn wc_lpc_destroy(l: *mut wc_lpc);
    pub fn wc_lpc_num_params(l: *const wc_lpc) -> u64;
    pub fn wc_lpc_set_params(l: *mut wc_lpc, params: *const f32, n: u64) -> wc_status;
    pub fn wc_lpc_get_params(l: *mut wc_lpc, params: *mut f32, n: u64) -> wc_status;
    pub fn wc_lpc_set_rounding(l: *mut wc_lpc, bf16: i32) -> wc_status;
    pub fn wc_lpc_forward_backward(l: *mut wc_lpc, n: i32, h: i32, w: i32, x: *const f32,
                                   feat: *const f32, dy: *const f32, y: *mut f32, grad: *mut f32,
                                   dx: *mut f32) -> wc_status;
    pub fn wc_lpc_forward(l: *mut wc_lpc, n: i32, h: i32, w: i32, x: *const f32, feat: *const f32,
                          tensor: i32, y: *mut f32) -> wc_status;
    pub fn wc_lpc_loss_grad(l: *mut wc_lpc, n: i32, h: i32, w: i32, c: *const f32,
                            heff: *const f32, bed: *const f32, e: *const f32, dx: f64, dy: f64,
                            loss: *mut f64, grad: *mut f32) -> wc_status;
    pub fn wc_lpc_harvest(l: *mut wc_lpc, s: *mut wc_solver) -> wc_status;
    pub fn wc_lpc_num_systems(l: *const wc_lpc) -> u64;
    pub fn wc_lpc_train(l: *mut wc_lpc, steps: u32, batch: u32, patch: u32, lr: f32, rough: f32,
                        seed: u64, losses: *mut f64) -> wc_status;
    pub fn wc_solver_set_lpc(s: *mut wc_solver, l: *mut wc_lpc) -> wc_status;

    // Per-step statistics and frames (crates/wavesim/src/lib.rs).
    pub fn wc_recorder_create(s: *mut wc_solver, from: f64, period: f64,
                              out: *mut *mut wc_recorder) -> wc_status;
    pub fn wc_recorder_destroy(r: *mut wc_recorder);
    pub fn wc_recorder_read(r: *mut wc_recorder, summary: *mut wc_record_summary,
                            eta_max: *mut f64, eta_min: *mut f64, wave_height: *mut f64,
                            breaking_fraction: *mut f64, harmonic: *mut f64) -> wc_status;
    pub fn wc_frame(s: *mut wc_solver, tide: f64, eta: *mut f32, breaking: *mut f32,
                    rise: *mut f64) -> wc_status;

    // One-way nesting.
    pub fn wc_nest_create(fine: *mut wc_solver, coarse: *mut wc_solver, zones: *const wc_sponge,
                          n_zones: u64, x_offset_m: f64, y_offset_m: f64,
                          out: *mut *mut wc_nest) -> wc_status;
    pub fn wc_nest_destroy(n: *mut wc_nest);
    pub fn wc_nest_cells(n: *const wc_nest) -> u64;
    pub fn wc_nest_sample(n: *mut wc_nest, slot: i32) -> wc_status;
    pub fn wc_nest_step(n: *mut wc_nest, dt: f64) -> wc_status;

    pub fn wc_launch_count(s: *const wc_solver) -> u64;
    pub fn wc_last_error() -> *const c_char;
}
