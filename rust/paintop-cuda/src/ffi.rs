//! Raw binding of include/paintop_cuda.h: every struct field for field and
//! every function parameter for parameter, in the header's order and C types.
#![allow(unsafe_code, non_camel_case_types, dead_code)]
use std::os::raw::{c_char, c_int, c_void};

pub type pt_status = c_int;
pub const PT_OK: pt_status = 0;
pub const PT_NO_DEVICE: pt_status = 1;
pub const PT_INVALID_ARG: pt_status = 2;
pub const PT_LAUNCH_FAILED: pt_status = 3;
pub const PT_TIMEOUT: pt_status = 4;
pub const PT_OOM: pt_status = 5;
pub const PT_INTERNAL: pt_status = 6;

pub const PT_FLAG_WARM_START: u32 = 0x1;
pub const PT_FLAG_DEVICE_POINTERS: u32 = 0x2;
pub const PT_FLAG_OMEGA_AUTO: u32 = 0x4;
pub const PT_FLAG_MULTIGRID: u32 = 0x8;

pub const PT_STOP_CONVERGED: i32 = 0;
pub const PT_STOP_MAX_ITERATIONS: i32 = 1;
pub const PT_STOP_STALLED: i32 = 2;

pub const PT_FILL_NONZERO: i32 = 0;
pub const PT_FILL_EVEN_ODD: i32 = 1;

pub const PT_KIND_IMAGE: u32 = 0;
pub const PT_KIND_MASK: u32 = 1;

pub const PT_NOALLOC_SCRATCH_BYTES: u32 = 64 * 1024 * 1024;

#[repr(C)] pub struct pt_ctx { _p: [u8; 0] }
#[repr(C)] pub struct pt_unet { _p: [u8; 0] }

#[repr(C)] pub struct pt_problem {
    pub width: u32, pub height: u32, pub channels: u32,
    pub source_or_guidance: *const f32, pub target_or_anchor: *const f32,
    pub mask: *const f32, pub lambda: f64, pub max_iterations: u32,
    pub tolerance: f64, pub omega: f64, pub flags: u32,
    pub initial_guess: *const f32,
}
#[repr(C)] pub struct pt_report {
    pub iterations: u32, pub converged: i32, pub stop_reason: i32,
    pub tolerance: f64, pub final_residual: f64, pub history_len: u32,
    pub omega_used: f64, pub refinements: u32, pub channel: i32,
    pub initial_residual: f64, pub warm_start: i32,
}
#[repr(C)] pub struct pt_port {
    pub name: *const c_char, pub kind: u32, pub width: u32, pub height: u32,
    pub channels: u32, pub samples: *const f32, pub sample_count: usize,
}
#[repr(C)] pub struct pt_error {
    pub error_class: [c_char; 16], pub code: [c_char; 40],
    pub message: [c_char; 256], pub actual: [c_char; 96],
}
#[repr(C)] pub struct pt_solver_data {
    pub kind: [c_char; 24], pub steps: u32, pub stability_number: f64,
    pub stability_limit: f64, pub stable: i32, pub total_energy: f64, pub iterations: u32,
    pub stop_reason: i32, pub converged: i32, pub tolerance: f64, pub final_residual: f64,
    pub history_len: u32,
}

unsafe extern "C" {
    pub fn pt_ctx_create(device: c_int, out: *mut *mut pt_ctx) -> pt_status;
    pub fn pt_ctx_destroy(ctx: *mut pt_ctx) -> pt_status;
    pub fn pt_poisson_solve(ctx: *mut pt_ctx, p: *const pt_problem, out_candidate: *mut f32,
        reports: *mut pt_report, history: *mut f64) -> pt_status;
    pub fn pt_poisson_solve_batch(ctx: *mut pt_ctx, ps: *const pt_problem, n: u32,
        outs: *const *mut f32, reports: *const *mut pt_report, histories: *const *mut f64) -> pt_status;
    pub fn pt_mask_ellipse(ctx: *mut pt_ctx, width: u32, height: u32, center_x: f64, center_y: f64,
        radius_x: f64, radius_y: f64, angle_rad: f64, half_width_px: f64, mask: *mut f32,
        flags: u32) -> pt_status;
    pub fn pt_mask_polygon(ctx: *mut pt_ctx, width: u32, height: u32, points_xy: *const f64,
        n_points: u32, fill_rule: i32, mask: *mut f32, flags: u32) -> pt_status;
    pub fn pt_op_compute(ctx: *mut pt_ctx, op_id: *const c_char, inputs: *const pt_port,
        n_inputs: u32, params_json: *const c_char, candidate: *mut f32, candidate_count: usize,
        solver: *mut pt_solver_data, residual_history: *mut f64, history_cap: u32,
        all_finite: *mut i32, err: *mut pt_error) -> pt_status;
    pub fn pt_op_compute_ex(ctx: *mut pt_ctx, op_id: *const c_char, inputs: *const pt_port,
        n_inputs: u32, params_json: *const c_char, candidate: *mut f32, candidate_count: usize,
        solver: *mut pt_solver_data, residual_history: *mut f64, history_cap: u32,
        all_finite: *mut i32, err: *mut pt_error, solve_flags: u32) -> pt_status;
    pub fn pt_status_str(s: pt_status) -> *const c_char;
    pub fn pt_ctx_last_error(ctx: *const pt_ctx) -> *const c_char;
    pub fn pt_ctx_set_budget(ctx: *mut pt_ctx, seconds: f64) -> pt_status;
    pub fn pt_ctx_stream(ctx: *const pt_ctx) -> *mut c_void;
    pub fn pt_ctx_last_timing(ctx: *const pt_ctx, solve_kernel_ms: *mut f64, call_ms: *mut f64,
        kernel_launches: *mut i64) -> pt_status;
    pub fn pt_ctx_last_transfer(ctx: *const pt_ctx, h2d_bytes: *mut u64, d2h_bytes: *mut u64) -> pt_status;
    pub fn pt_tile_config_count() -> u32;
    pub fn pt_tile_config_info(idx: u32, sweeps_per_step: *mut i32, tile_w: *mut i32,
        tile_h: *mut i32) -> pt_status;
    pub fn pt_ctx_set_config(ctx: *mut pt_ctx, cfg: i32) -> pt_status;
    pub fn pt_ctx_last_config(ctx: *const pt_ctx) -> i32;
    pub fn pt_autotune(ctx: *mut pt_ctx, ps: *const pt_problem, n: u32, repeats: u32,
        outs: *const *mut f32, reports: *const *mut pt_report, chosen: *mut i32,
        ms_per_config: *mut f64) -> pt_status;
    pub fn pt_poisson_solve_noalloc(p: *const pt_problem, out_candidate: *mut f32,
        reports: *mut pt_report, history: *mut f64, stream: *mut c_void) -> pt_status;
    pub fn pt_unet_create(ctx: *mut pt_ctx, seed: u64, out: *mut *mut pt_unet) -> pt_status;
    pub fn pt_unet_destroy(net: *mut pt_unet) -> pt_status;
    pub fn pt_unet_param_count(net: *const pt_unet) -> u64;
    pub fn pt_unet_get_params(net: *mut pt_unet, host: *mut f32) -> pt_status;
    pub fn pt_unet_set_params(net: *mut pt_unet, host: *const f32) -> pt_status;
    pub fn pt_unet_features(net: *mut pt_unet, guidance: *const f32, anchor: *const f32,
        mask: *const f32, batch: u32, h: u32, w: u32, features: *mut f32) -> pt_status;
    pub fn pt_unet_forward(net: *mut pt_unet, features: *const f32, batch: u32, h: u32, w: u32,
        pred: *mut f32) -> pt_status;
    pub fn pt_unet_loss_grad(net: *mut pt_unet, features: *const f32, target: *const f32,
        loss_mask: *const f32, batch: u32, h: u32, w: u32, loss: *mut f64, grad_host: *mut f32) -> pt_status;
    pub fn pt_unet_train_step(net: *mut pt_unet, features: *const f32, target: *const f32,
        loss_mask: *const f32, batch: u32, h: u32, w: u32, lr: f32, loss: *mut f64) -> pt_status;
    pub fn pt_unet_grad_record(net: *mut pt_unet, features: *const f32, target: *const f32,
        loss_mask: *const f32, batch: u32, h: u32, w: u32, loss: *mut f64, record: *mut f32) -> pt_status;
    pub fn pt_unet_apply_records(net: *mut pt_unet, records: *const f32, replicas: u32,
        lr: f32) -> pt_status;
    pub fn pt_unet_guess(net: *mut pt_unet, guidance: *const f32, anchor: *const f32,
        mask: *const f32, width: u32, height: u32, channels: u32, scale: u32,
        guess: *mut f32) -> pt_status;
    pub fn pt_unet_save(net: *mut pt_unet, path: *const c_char) -> pt_status;
    pub fn pt_unet_load(net: *mut pt_unet, path: *const c_char) -> pt_status;
}

/// One device context per process, created on first use. The library
/// serialises calls on a context, so one context may be shared by threads.
pub struct Ctx(*mut pt_ctx);
unsafe impl Send for Ctx {}
unsafe impl Sync for Ctx {}
impl Ctx {
    pub fn new(device: i32) -> Result<Self, pt_status> {
        let mut h = std::ptr::null_mut();
        let st = unsafe { pt_ctx_create(device, &mut h) };
        if st == PT_OK { Ok(Ctx(h)) } else { Err(st) }
    }
    pub fn raw(&self) -> *mut pt_ctx { self.0 }
}
impl Drop for Ctx {
    fn drop(&mut self) { unsafe { pt_ctx_destroy(self.0); } }
}

/// A NUL-terminated fixed-size C string field as a Rust string.
pub fn field_str(a: &[c_char]) -> String {
    let bytes: Vec<u8> = a.iter().take_while(|&&c| c != 0).map(|&c| c as u8).collect();
    String::from_utf8_lossy(&bytes).into_owned()
}
