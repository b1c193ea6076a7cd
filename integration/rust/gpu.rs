//! FFI declarations of the B200 fitness-evaluation engine (`include/rsr_gpu.h`)
//! for rsr's Rust crate: this file goes to `src/engine/ffi/gpu.rs`, next to the
//! existing SymEngine binding (`src/engine/ffi/symengine.rs:4-6`), and
//! `build.rs` links `librsrgpu.so` (see `build.rs` in this directory).
//!
//! Every `extern "C"` function below is one `RSR_API` entry point of the
//! header, with the same name and parameter types; every `#[repr(C)]` struct
//! mirrors the header's struct field for field, in order.  Status codes are
//! the header's `rsr_status` values.
#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_int};

// ------------------------------------------------------------ rsr_status
pub const RSR_OK: c_int = 0;
pub const RSR_EINVAL: c_int = 1;
pub const RSR_EPROGRAM: c_int = 2;
pub const RSR_ENOMEM: c_int = 3;
pub const RSR_ENODEV: c_int = 4;
pub const RSR_ECUDA: c_int = 5;
pub const RSR_ETIMEDOUT: c_int = 6;
pub const RSR_ENOTFOUND: c_int = 7;
pub const RSR_EBUSY: c_int = 8;
pub const RSR_ECANCELED: c_int = 9;

// ------------------------------------------------------------ rsr_kernel
pub const RSR_KERNEL_AUTO: c_int = 0;
pub const RSR_KERNEL_PLAIN: c_int = 1;
pub const RSR_KERNEL_BATCHED: c_int = 2;

pub const RSR_OPT_NO_LOAD_FUSION: u32 = 1;
pub const RSR_OPT_SLOT_ADJOINT: u32 = 2;

// --------------------------------------------------------- rsr_job_kind
pub const RSR_JOB_MSE: u32 = 0;
pub const RSR_JOB_MSE_GRAD: u32 = 1;
pub const RSR_JOB_FIT: u32 = 2;
pub const RSR_JOB_FIT_AUTO: u32 = 3;

// -------------------------------------------------------- rsr_job_state
pub const RSR_JOB_QUEUED: u32 = 0;
pub const RSR_JOB_RUNNING: u32 = 1;
pub const RSR_JOB_DONE: u32 = 2;

/// Handle of a resident dataset (`rsr_dataset`).
pub type RsrDataset = u64;

/// Opaque engine context (`rsr_ctx`).
#[repr(C)]
pub struct RsrCtx {
    _private: [u8; 0],
}

/// Opaque serving loop (`rsr_server`).
#[repr(C)]
pub struct RsrServer {
    _private: [u8; 0],
}

/// Opaque prepared batch (`rsr_batch`).
#[repr(C)]
pub struct RsrBatch {
    _private: [u8; 0],
}

/// One compiled `Program` (`program.rs:18-23`): code words, constant kinds,
/// flattened parameters.
#[repr(C)]
pub struct RsrProgram {
    pub code: *const u32,
    pub len: u32,
    pub const_kinds: *const u8,
    pub n_consts: u32,
    pub params: *const f32,
    pub n_params: u32,
}

/// A population in concatenated arrays; the `*_off` arrays hold
/// `n_programs + 1` element offsets.
#[repr(C)]
pub struct RsrPopulation {
    pub n_programs: u32,
    pub code: *const u32,
    pub code_off: *const u64,
    pub const_kinds: *const u8,
    pub kind_off: *const u64,
    pub params: *const f32,
    pub param_off: *const u64,
}

#[repr(C)]
pub struct RsrOptions {
    pub struct_size: u32,
    pub kernel: i32,
    pub points_per_thread: i32,
    pub programs_per_warp: i32,
    pub use_graphs: i32,
    pub mem_budget_bytes: u64,
    pub tune_cache_path: *const c_char,
    pub flags: u32,
}

#[repr(C)]
pub struct RsrFitStats {
    pub iterations: u32,
    pub gradient_evaluations: u32,
    pub mse_evaluations: u32,
}

#[repr(C)]
pub struct RsrServerOptions {
    pub struct_size: u32,
    pub slots: u32,
    pub max_batch_programs: u32,
    pub max_queue: u32,
    pub mem_budget_bytes: u64,
}

#[repr(C)]
pub struct RsrJob {
    pub kind: u32,
    pub fit_iterations: u32,
    pub pop: *const RsrPopulation,
    pub ds: RsrDataset,
    pub ds_per_program: *const RsrDataset,
    pub mse_out: *mut f32,
    pub grad_out: *mut f32,
    pub params_out: *mut f32,
    pub seed: u64,
}

#[repr(C)]
pub struct RsrJobInfo {
    pub status: i32,
    pub batch_jobs: u32,
    pub queue_ms: f64,
    pub latency_ms: f64,
}

#[repr(C)]
pub struct RsrServingStats {
    pub submitted: u64,
    pub completed: u64,
    pub failed: u64,
    pub cancelled: u64,
    pub refused: u64,
    pub launches: u64,
    pub peak_mem_bytes: u64,
    pub p50_ms: f64,
    pub p95_ms: f64,
    pub p99_ms: f64,
    pub mean_ms: f64,
    pub max_ms: f64,
    pub program_points_per_sec: f64,
    pub wall_s: f64,
}

#[repr(C)]
pub struct RsrProgramInfo {
    pub depth_ref: [u32; 5],
    pub depth_fast: [u32; 5],
    pub n_uops_fast: u32,
    pub n_uops_plain: u32,
    pub fast_profile: i32,
    pub flops_per_point: u32,
}

extern "C" {
    // ------------------------------------------------------------ context
    pub fn rsr_options_default(opts: *mut RsrOptions);
    pub fn rsr_ctx_create(device: c_int, opts: *const RsrOptions, out: *mut *mut RsrCtx) -> c_int;
    pub fn rsr_ctx_destroy(ctx: *mut RsrCtx) -> c_int;
    pub fn rsr_last_error() -> *const c_char;
    pub fn rsr_version() -> *const c_char;

    // ----------------------------------------------------------- datasets
    pub fn rsr_dataset_upload(ctx: *mut RsrCtx, feature_flat: *const f32, target_batches: *const f32,
                              num_features: u32, num_batches: u64, num_samples: u64,
                              out: *mut RsrDataset) -> c_int;
    pub fn rsr_dataset_upload_columns(ctx: *mut RsrCtx, features: *const f32, targets: *const f32,
                                      num_features: u32, n: u64, out: *mut RsrDataset) -> c_int;
    pub fn rsr_dataset_upload_rows(ctx: *mut RsrCtx, x_rows: *const f32, y: *const f32, num_features: u32,
                                   num_samples: u64, normalize: c_int, stats_out: *mut f32,
                                   out: *mut RsrDataset) -> c_int;
    pub fn rsr_dataset_subset(ctx: *mut RsrCtx, src: RsrDataset, target_samples: u64,
                              out: *mut RsrDataset) -> c_int;
    pub fn rsr_dataset_download(ctx: *mut RsrCtx, ds: RsrDataset, feature_flat: *mut f32,
                                target_batches: *mut f32) -> c_int;
    pub fn rsr_dataset_release(ctx: *mut RsrCtx, ds: RsrDataset) -> c_int;
    pub fn rsr_dataset_info(ctx: *mut RsrCtx, ds: RsrDataset, num_features: *mut u32, num_batches: *mut u64,
                            num_samples: *mut u64) -> c_int;

    // ------------------------------------------------ reference drop-ins
    pub fn rsr_compute_mse(ctx: *mut RsrCtx, prog: *const RsrProgram, ds: RsrDataset, mse: *mut f32) -> c_int;
    pub fn rsr_compute_mse_with_gradient(ctx: *mut RsrCtx, prog: *const RsrProgram, ds: RsrDataset,
                                         mse: *mut f32, grad: *mut f32) -> c_int;
    pub fn rsr_eval_points(ctx: *mut RsrCtx, prog: *const RsrProgram, ds: RsrDataset, out: *mut f32) -> c_int;

    // ------------------------------------------------------------ batched
    pub fn rsr_eval_mse_batch(ctx: *mut RsrCtx, pop: *const RsrPopulation, ds: RsrDataset,
                              ds_per_program: *const RsrDataset, kernel: c_int, mse_out: *mut f32) -> c_int;
    pub fn rsr_eval_mse_grad_batch(ctx: *mut RsrCtx, pop: *const RsrPopulation, ds: RsrDataset,
                                   ds_per_program: *const RsrDataset, mse_out: *mut f32,
                                   grad_out: *mut f32) -> c_int;
    pub fn rsr_eval_points_batch(ctx: *mut RsrCtx, pop: *const RsrPopulation, ds: RsrDataset, kernel: c_int,
                                 out: *mut f32) -> c_int;
    pub fn rsr_compute_mse_noalloc(ctx: *mut RsrCtx, prog: *const RsrProgram, ds: RsrDataset,
                                   mse: *mut f32) -> c_int;
    pub fn rsr_eval_sums_batch(ctx: *mut RsrCtx, pop: *const RsrPopulation, ds: RsrDataset,
                               ds_per_program: *const RsrDataset, gradient: c_int, sums_out: *mut f64) -> c_int;
    pub fn rsr_finalize_sums(n: u32, gradient: c_int, sums: *const f64, num_samples: u64, mse_out: *mut f32,
                             grad_out: *mut f32) -> c_int;

    // --------------------------------------------------- constant fitting
    pub fn rsr_fit_lbfgs(ctx: *mut RsrCtx, pop: *const RsrPopulation, ds: RsrDataset,
                         ds_per_program: *const RsrDataset, max_iterations: u32, params_out: *mut f32,
                         mse_out: *mut f32, stats: *mut RsrFitStats) -> c_int;
    pub fn rsr_fit_nelder_mead(ctx: *mut RsrCtx, pop: *const RsrPopulation, ds: RsrDataset,
                               ds_per_program: *const RsrDataset, max_iterations: u32, params_out: *mut f32,
                               mse_out: *mut f32, stats: *mut RsrFitStats) -> c_int;
    pub fn rsr_fit_cma_es(ctx: *mut RsrCtx, pop: *const RsrPopulation, ds: RsrDataset,
                          ds_per_program: *const RsrDataset, max_iterations: u32, seed: u64, params_out: *mut f32,
                          mse_out: *mut f32, stats: *mut RsrFitStats) -> c_int;

    // ------------------------------------------------------------ serving
    pub fn rsr_server_options_default(opts: *mut RsrServerOptions);
    pub fn rsr_server_create(ctx: *mut RsrCtx, opts: *const RsrServerOptions, out: *mut *mut RsrServer) -> c_int;
    pub fn rsr_server_destroy(srv: *mut RsrServer) -> c_int;
    pub fn rsr_submit(srv: *mut RsrServer, job: *const RsrJob, ticket: *mut u64) -> c_int;
    pub fn rsr_poll(srv: *mut RsrServer, ticket: u64, state: *mut u32) -> c_int;
    pub fn rsr_wait(srv: *mut RsrServer, ticket: u64, timeout_us: u64, info: *mut RsrJobInfo) -> c_int;
    pub fn rsr_cancel(srv: *mut RsrServer, ticket: u64) -> c_int;
    pub fn rsr_server_stats(srv: *mut RsrServer, stats: *mut RsrServingStats, reset: c_int) -> c_int;

    // --------------------------------------------------- prepared batches
    pub fn rsr_batch_prepare(ctx: *mut RsrCtx, pop: *const RsrPopulation, ds: RsrDataset,
                             ds_per_program: *const RsrDataset, kernel: c_int, with_gradient: c_int,
                             out: *mut *mut RsrBatch) -> c_int;
    pub fn rsr_batch_run(ctx: *mut RsrCtx, b: *mut RsrBatch) -> c_int;
    pub fn rsr_batch_results(ctx: *mut RsrCtx, b: *mut RsrBatch, mse_out: *mut f32, grad_out: *mut f32) -> c_int;
    pub fn rsr_batch_last_timing(ctx: *mut RsrCtx, b: *mut RsrBatch, eval_ms: *mut f32,
                                 total_ms: *mut f32) -> c_int;
    pub fn rsr_batch_describe(ctx: *mut RsrCtx, b: *mut RsrBatch, buf: *mut c_char, buf_len: usize) -> c_int;
    pub fn rsr_batch_destroy(ctx: *mut RsrCtx, b: *mut RsrBatch) -> c_int;

    // ------------------------------------------- tuning and measurement
    pub fn rsr_autotune(ctx: *mut RsrCtx, pop: *const RsrPopulation, ds: RsrDataset,
                        ds_per_program: *const RsrDataset, reps: c_int, report: *mut c_char,
                        report_len: usize) -> c_int;
    pub fn rsr_ctx_launch_count(ctx: *mut RsrCtx) -> u64;
    pub fn rsr_ctx_last_transfer(ctx: *mut RsrCtx, h2d_bytes: *mut u64, d2h_bytes: *mut u64) -> c_int;
    pub fn rsr_flush_l2(ctx: *mut RsrCtx) -> c_int;
    pub fn rsr_synchronize(ctx: *mut RsrCtx) -> c_int;
    pub fn rsr_measure_fp32_peak(ctx: *mut RsrCtx, lane_ops_per_s: *mut f64) -> c_int;

    // ------------------------------------------------------ host encoder
    pub fn rsr_validate_program(prog: *const RsrProgram, num_features: u32) -> c_int;
    pub fn rsr_program_analyze(prog: *const RsrProgram, num_features: u32, info: *mut RsrProgramInfo) -> c_int;
    pub fn rsr_program_encoding(prog: *const RsrProgram, num_features: u32, form: c_int, out: *mut u32, cap: u32,
                                len: *mut u32) -> c_int;
}

/// The legacy evaluator API is infallible: a non-zero status becomes a panic
/// carrying the engine's message.
pub fn check(status: c_int) {
    if status != RSR_OK {
        let msg = unsafe { std::ffi::CStr::from_ptr(rsr_last_error()) };
        panic!("rsr-b200 engine error {}: {}", status, msg.to_string_lossy());
    }
}
