/*
 * rsr_gpu.h -- C ABI of the B200 fitness-evaluation engine for rsr.
 *
 * The engine replaces rsr's CPU evaluator (src/engine/eval/evaluator.rs) behind
 * plain pointers and sizes.  Every entry point returns an rsr_status; 0 is
 * success and rsr_last_error() describes the last failure on the calling
 * thread.  All host buffers are caller-owned and only read (or written, for
 * outputs) during the call; nothing is retained unless stated.
 *
 * Program format (the reference's compiled Program, src/engine/expr/program.rs:18-23):
 *   code[i]        one word per Instruction: opcode | operand << 8.  Opcodes
 *                  follow the variant order of compose_engine!
 *                  (src/engine/domain.rs:46-63) then BasicOpCode
 *                  (src/domains/basic/mod.rs:9-20) then LinalgOpCode
 *                  (src/domains/linalg/mod.rs:9-51).  The operand is the
 *                  feature offset of LoadVar* or the constant index of
 *                  LoadConst*.
 *   const_kinds[c] Scalar variant of constant c (src/engine/eval/scalar.rs:4-12):
 *                  0 Float, 1 Int, 2 Bool, 3 Vec2, 4 Vec3, 5 Mat2, 6 Mat3.
 *   params         the flattened constants, Parameterized::flatten_params
 *                  order (src/engine/expr/program.rs:100-145).
 *
 * Dataset format (src/engine/data/dataset.rs:18-34): feature_flat holds
 * num_batches*num_features groups of 8 floats (f32x8), group b*F+f carrying
 * feature f of points 8b..8b+7; target_batches holds num_batches groups of 8.
 * Padded lanes are evaluated and counted, the divisor is num_samples, exactly
 * as compute_mse does (evaluator.rs:159-173).
 */
#ifndef RSR_GPU_H
#define RSR_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RSR_API __attribute__((visibility("default")))
#else
#define RSR_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rsr_status {
    RSR_OK = 0,
    RSR_EINVAL = 1,      /* bad argument or handle */
    RSR_EPROGRAM = 2,    /* malformed program: unknown opcode, stack underflow,
                            more than 32 slots on a stack, index out of range */
    RSR_ENOMEM = 3,      /* device or host allocation failed */
    RSR_ENODEV = 4,      /* no usable sm_100 device */
    RSR_ECUDA = 5,       /* CUDA runtime error */
    RSR_ETIMEDOUT = 6,   /* a bounded wait expired */
    RSR_ENOTFOUND = 7,   /* unknown dataset handle or ticket */
    RSR_EBUSY = 8,       /* admission refused (memory budget or queue full) */
    RSR_ECANCELED = 9    /* job cancelled or server shut down */
} rsr_status;

typedef struct rsr_ctx rsr_ctx;
typedef uint64_t rsr_dataset;

typedef struct rsr_program {
    const uint32_t *code;
    uint32_t len;
    const uint8_t *const_kinds;
    uint32_t n_consts;
    const float *params;
    uint32_t n_params;
} rsr_program;

/* A population packed into concatenated arrays; *_off have n_programs+1
 * entries (element offsets). */
typedef struct rsr_population {
    uint32_t n_programs;
    const uint32_t *code;
    const uint64_t *code_off;
    const uint8_t *const_kinds;
    const uint64_t *kind_off;
    const float *params;
    const uint64_t *param_off;
} rsr_population;

/* Kernel selection for evaluation calls. */
typedef enum rsr_kernel {
    RSR_KERNEL_AUTO = 0,     /* register-stack batched kernel where a program fits, slot-file kernel otherwise */
    RSR_KERNEL_PLAIN = 1,    /* slot-file interpreter, one program per warp, single launch */
    RSR_KERNEL_BATCHED = 2   /* register-stack persistent kernel (programs that do not fit fall back to PLAIN) */
} rsr_kernel;

typedef struct rsr_options {
    uint32_t struct_size;        /* sizeof(rsr_options) */
    int32_t kernel;              /* rsr_kernel */
    int32_t points_per_thread;   /* 0 = autotuned; else 1, 2, 4 or 8 */
    int32_t programs_per_warp;   /* 0 = autotuned; else 1..8 */
    int32_t use_graphs;          /* replay prepared batches through CUDA graphs */
    uint64_t mem_budget_bytes;   /* 0 = 90% of free device memory at creation */
    const char *tune_cache_path; /* autotuner cache (JSON); NULL = in memory only */
    uint32_t flags;              /* RSR_OPT_* */
} rsr_options;

/* rsr_options.flags */
#define RSR_OPT_NO_LOAD_FUSION 1u   /* register kernel: keep loads as separate micro-ops */
#define RSR_OPT_SLOT_ADJOINT 2u     /* gradients: the slot-file adjoint for every program (else the
                                       register adjoint where a program fits it) */

/* ------------------------------------------------------------- context */
RSR_API void rsr_options_default(rsr_options *opts);
RSR_API int rsr_ctx_create(int device, const rsr_options *opts, rsr_ctx **out);
RSR_API int rsr_ctx_destroy(rsr_ctx *ctx);
RSR_API const char *rsr_last_error(void);
RSR_API const char *rsr_version(void);

/* ------------------------------------------------------------ datasets */
/* Upload a Dataset (dataset.rs:18-34 fields) and keep it resident.  Replaces
 * the per-call &Dataset borrow of compute_mse (evaluator.rs:153). */
RSR_API int rsr_dataset_upload(rsr_ctx *ctx, const float *feature_flat, const float *target_batches,
                       uint32_t num_features, uint64_t num_batches, uint64_t num_samples, rsr_dataset *out);
/* Same dataset given as columns: features[f*n + i], targets[i], i < n; padded
 * to a multiple of 8 with zeros as Dataset::new does (dataset.rs:96-154). */
RSR_API int rsr_dataset_upload_columns(rsr_ctx *ctx, const float *features, const float *targets, uint32_t num_features,
                               uint64_t n, rsr_dataset *out);
/* Dataset::new (src/engine/data/dataset.rs:37-169) on the device: raw rows
 * x_rows[num_samples][num_features] and y[num_samples]; with normalize != 0
 * every column is z-scored with the reference's sequential f32 sums (means,
 * deviations and normalised values bit-identical to the reference's).
 * stats_out (optional, 2*(num_features+1) floats): the feature means then the
 * target mean, the feature deviations then the target deviation. */
RSR_API int rsr_dataset_upload_rows(rsr_ctx *ctx, const float *x_rows, const float *y, uint32_t num_features,
                                    uint64_t num_samples, int normalize, float *stats_out, rsr_dataset *out);
/* Dataset::subset (dataset.rs:360-447) of a resident dataset, as a new
 * resident dataset: min(target_samples, num_samples) evenly spaced points
 * (the engine's mini-batch, src/engine/search/engine.rs:49). */
RSR_API int rsr_dataset_subset(rsr_ctx *ctx, rsr_dataset src, uint64_t target_samples, rsr_dataset *out);
/* A resident dataset back in the AoSoA layout: feature_flat
 * [num_batches*num_features*8], target_batches [num_batches*8]. */
RSR_API int rsr_dataset_download(rsr_ctx *ctx, rsr_dataset ds, float *feature_flat, float *target_batches);
RSR_API int rsr_dataset_release(rsr_ctx *ctx, rsr_dataset ds);
RSR_API int rsr_dataset_info(rsr_ctx *ctx, rsr_dataset ds, uint32_t *num_features, uint64_t *num_batches,
                     uint64_t *num_samples);

/* ------------------------------------------------- reference drop-ins */
/* evaluator::compute_mse (src/engine/eval/evaluator.rs:153-174). */
RSR_API int rsr_compute_mse(rsr_ctx *ctx, const rsr_program *prog, rsr_dataset ds, float *mse);
/* evaluator::compute_mse_with_gradient (evaluator.rs:177-224): mse and
 * grad[32], d(MSE)/d(flat parameter k) for k < min(param_count, 32), zeros
 * elsewhere; non-finite MSE gives (f32::MAX, zeros). */
RSR_API int rsr_compute_mse_with_gradient(rsr_ctx *ctx, const rsr_program *prog, rsr_dataset ds, float *mse, float *grad);
/* evaluator::eval_simd (evaluator.rs:20-150) applied to every batch of the
 * dataset: out[num_batches*8] predictions, padded lanes included. */
RSR_API int rsr_eval_points(rsr_ctx *ctx, const rsr_program *prog, rsr_dataset ds, float *out);

/* ------------------------------------------------------------- batched */
/* compute_mse for a whole population against one dataset (ds_per_program
 * NULL) or against ds_per_program[i]. */
RSR_API int rsr_eval_mse_batch(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *ds_per_program,
                       int kernel, float *mse_out);
/* compute_mse_with_gradient for a population: mse_out[n], grad_out[n*32]. */
RSR_API int rsr_eval_mse_grad_batch(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds,
                            const rsr_dataset *ds_per_program, float *mse_out, float *grad_out);
/* eval_simd over every batch for each program: out[i*num_batches*8 + j]. */
RSR_API int rsr_eval_points_batch(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, int kernel, float *out);

/* rsr_compute_mse without allocation.  No reference counterpart: an extra
 * entry point for callers that must not allocate device memory per call --
 * a serving loop whose device memory is all handed out to a fixed pool (a
 * cudaMalloc there fails or evicts), or a host thread that shares the GPU
 * with running streams (cudaFree synchronises the whole device).
 * The slot-file kernel runs with its descriptors, code, constants, work
 * items and partial sums in one static device array of 256 KiB per device,
 * so the program is limited to 512 instructions and 1024 constants /
 * parameter floats, and the dataset to 16,777,216 points; larger inputs
 * return RSR_EINVAL.  The first call on a device takes the array's address
 * (cudaGetSymbolAddress, with the device current) and loads every kernel the
 * entry point launches (lazy module loading would otherwise allocate on a
 * kernel's first launch); it should come before any stream capture on that
 * device.  Calls after it allocate no device memory.  Calls that overlap in time on one device
 * through different contexts race on the array.  The dataset must already
 * be resident (rsr_dataset_upload). */
RSR_API int rsr_compute_mse_noalloc(rsr_ctx *ctx, const rsr_program *prog, rsr_dataset ds, float *mse);

/* Point sharding (a dataset split across GPUs by 8-point batches, the last
 * shard holding the padding): per-program unscaled f64 sums of one shard --
 * SSE, or SSE followed by the 32 gradient sums when gradient != 0
 * (n x 33 doubles) -- in caller order.  The shards' sums are added (one
 * all-reduce) and rsr_finalize_sums applies the epilogue of compute_mse /
 * compute_mse_with_gradient (evaluator.rs:172-173, 211-223) with the whole
 * dataset's num_samples. */
RSR_API int rsr_eval_sums_batch(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds,
                                const rsr_dataset *ds_per_program, int gradient, double *sums_out);
RSR_API int rsr_finalize_sums(uint32_t n, int gradient, const double *sums, uint64_t num_samples, float *mse_out,
                              float *grad_out);

/* ----------------------------------------------------- constant fitting */
typedef struct rsr_fit_stats {
    uint32_t iterations;            /* L-BFGS iterations taken by the slowest program */
    uint32_t gradient_evaluations;  /* batched gradient launches */
    uint32_t mse_evaluations;       /* batched line-search launches */
} rsr_fit_stats;
/* run_lbfgs (src/engine/optimize/lbfgs.rs:9-165) for a whole population:
 * up to max_iterations L-BFGS steps per program (memory 6, at most 32
 * parameters, Armijo backtracking c1 = 1e-4 with up to 11 halvings, stop at
 * |grad| < 1e-5), gradients from the adjoint kernel, line-search MSEs from
 * the register kernel.  params_out (same layout as pop->params) receives the
 * fitted constants, mse_out[i] the final fitness of program i. */
RSR_API int rsr_fit_lbfgs(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *ds_per_program,
                          uint32_t max_iterations, float *params_out, float *mse_out, rsr_fit_stats *stats);

/* ------------------------------------------------------------ serving
 * A device-resident request loop for the island threads (the callers of
 * Individual::calculate_mse, src/engine/search/island.rs:150-238, and of
 * optimize_individual_constants, src/engine/optimize/mod.rs:10-59): jobs are
 * submitted from any thread, datasets stay resident, and `slots` worker
 * streams keep several jobs on the device at once.  Continuous batching:
 * a free slot takes the oldest waiting job and merges the evaluation jobs of
 * the same kind queued behind it (up to max_batch_programs programs) into
 * one launch.  Memory admission: a job whose estimated device footprint is
 * above the budget is refused at submit (RSR_ENOMEM); otherwise it waits
 * until the running jobs' footprints leave room for it. */
typedef struct rsr_server rsr_server;

typedef struct rsr_server_options {
    uint32_t struct_size;
    uint32_t slots;               /* jobs on the device at once; default 4 */
    uint32_t max_batch_programs;  /* programs merged into one launch; default 16384 */
    uint32_t max_queue;           /* waiting jobs before submit returns RSR_EBUSY; default 65536 */
    uint64_t mem_budget_bytes;    /* device bytes of in-flight jobs; 0 = half the context's free budget */
} rsr_server_options;

typedef enum rsr_job_kind {
    RSR_JOB_MSE = 0,       /* mse_out[n] */
    RSR_JOB_MSE_GRAD = 1,  /* mse_out[n], grad_out[n*32] */
    RSR_JOB_FIT = 2,       /* rsr_fit_lbfgs: params_out (pop->params layout), mse_out[n] */
    /* optimize_individual_constants (src/engine/optimize/mod.rs:10-59) per
     * program: L-BFGS (15 iterations) for differentiable programs, CMA-ES
     * (max(fit_iterations / 16, 2) generations, streams from `seed`) for the
     * others with a vector or matrix constant, Nelder-Mead (fit_iterations)
     * otherwise; params_out and mse_out as RSR_JOB_FIT */
    RSR_JOB_FIT_AUTO = 3
} rsr_job_kind;

typedef struct rsr_job {
    uint32_t kind;                       /* rsr_job_kind */
    uint32_t fit_iterations;             /* RSR_JOB_FIT */
    const rsr_population *pop;           /* copied by rsr_submit */
    rsr_dataset ds;                      /* dataset of every program, unless ... */
    const rsr_dataset *ds_per_program;   /* ... one per program (copied) */
    float *mse_out;                      /* written when the job completes; */
    float *grad_out;                     /* the caller keeps these valid until */
    float *params_out;                   /* rsr_wait returns or the job is cancelled */
    uint64_t seed;                       /* RSR_JOB_FIT_AUTO: CMA-ES random streams */
} rsr_job;

typedef enum rsr_job_state { RSR_JOB_QUEUED = 0, RSR_JOB_RUNNING = 1, RSR_JOB_DONE = 2 } rsr_job_state;

typedef struct rsr_job_info {
    int32_t status;          /* rsr_status of the job */
    uint32_t batch_jobs;     /* jobs that shared its launch */
    double queue_ms;         /* submit -> taken by a slot */
    double latency_ms;       /* submit -> results written */
} rsr_job_info;

typedef struct rsr_serving_stats {
    uint64_t submitted, completed, failed, cancelled, refused;
    uint64_t launches;               /* batches run (merged launches count once) */
    uint64_t peak_mem_bytes;         /* largest admitted in-flight footprint */
    double p50_ms, p95_ms, p99_ms, mean_ms, max_ms;   /* latency of completed jobs */
    double program_points_per_sec;   /* completed program*points / busy wall time */
    double wall_s;                   /* first submit -> last completion */
} rsr_serving_stats;

RSR_API void rsr_server_options_default(rsr_server_options *opts);
RSR_API int rsr_server_create(rsr_ctx *ctx, const rsr_server_options *opts, rsr_server **out);
/* Cancels waiting jobs, finishes running ones, joins the workers. */
RSR_API int rsr_server_destroy(rsr_server *srv);
RSR_API int rsr_submit(rsr_server *srv, const rsr_job *job, uint64_t *ticket);
RSR_API int rsr_poll(rsr_server *srv, uint64_t ticket, uint32_t *state);
/* Waits up to timeout_us (0 = forever) and returns the job's status (the
 * ticket is then retired), or RSR_ETIMEDOUT leaving the job in place. */
RSR_API int rsr_wait(rsr_server *srv, uint64_t ticket, uint64_t timeout_us, rsr_job_info *info);
/* A waiting job is dropped; a running fit stops after its current step;
 * a running evaluation completes.  Wait on the ticket afterwards. */
RSR_API int rsr_cancel(rsr_server *srv, uint64_t ticket);
RSR_API int rsr_server_stats(rsr_server *srv, rsr_serving_stats *stats, int reset);

/* run_nelder_mead (src/engine/optimize/nelder_mead.rs:9-165) for a whole
 * population: a simplex over each program's Float constants (at most 32),
 * objective mse + 0.01 * sum |c|, up to max_iterations iterations; each
 * phase (reflection; expansion or contraction; each shrink vertex) is one
 * launch for all programs in it.  params_out gets the best vertex's
 * constants (other parameters unchanged), mse_out its MSE.  Vertices of
 * equal fitness keep their order (a stable sort; the reference's order for
 * ties is unspecified). */
RSR_API int rsr_fit_nelder_mead(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds,
                                const rsr_dataset *ds_per_program, uint32_t max_iterations, float *params_out,
                                float *mse_out, rsr_fit_stats *stats);

/* run_cma_es (src/engine/optimize/cmaes.rs:19-192) for a whole population,
 * the fit for non-differentiable programs with vector or matrix constants:
 * max_iterations generations of 16 candidates per program (best 8
 * recombined, diagonal covariance, sigma 0.5 shrinking by exp(-0.01), stop
 * when the best MSE < 1e-8), objective mse + 0.01 * sum |x| over the
 * reference's search vector (the flat parameters and a copy of them).  One
 * launch scores the 16 candidates of every program.  The reference draws from
 * an unseeded thread-local generator; here program i draws from a splitmix64
 * stream seeded from (seed, i), so a population's result does not depend on
 * its batching.  params_out receives the best point's parameters, mse_out[i]
 * its MSE (the starting MSE for programs without parameters). */
RSR_API int rsr_fit_cma_es(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *ds_per_program,
                           uint32_t max_iterations, uint64_t seed, float *params_out, float *mse_out,
                           rsr_fit_stats *stats);

/* -------------------------------------------------- prepared batches */
/* A population encoded and uploaded once, then run many times with inputs
 * resident on the device (the timed unit of the benchmark).  run() enqueues
 * the kernels on the context's stream (graph replay when enabled) and
 * returns without waiting; results() waits and copies mse back. */
typedef struct rsr_batch rsr_batch;
RSR_API int rsr_batch_prepare(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *ds_per_program,
                      int kernel, int with_gradient, rsr_batch **out);
RSR_API int rsr_batch_run(rsr_ctx *ctx, rsr_batch *b);
RSR_API int rsr_batch_results(rsr_ctx *ctx, rsr_batch *b, float *mse_out, float *grad_out);
/* Device time in milliseconds of the last run's kernels (CUDA events on the
 * launching stream), split into the evaluation kernels and the finalize. */
RSR_API int rsr_batch_last_timing(rsr_ctx *ctx, rsr_batch *b, float *eval_ms, float *total_ms);
/* Describes the prepared launch: kernel names used, points per thread,
 * programs per warp, number of work items, programs on the fallback path. */
RSR_API int rsr_batch_describe(rsr_ctx *ctx, rsr_batch *b, char *buf, size_t buf_len);
RSR_API int rsr_batch_destroy(rsr_ctx *ctx, rsr_batch *b);

/* Autotuner: times the register kernel's launch shapes (points per thread
 * 2/4/8, programs per warp 1/2/4/8) on this population and keeps the
 * fastest per kernel profile and dataset size class for later calls on the
 * context.  report (optional) receives the timings as JSON. */
RSR_API int rsr_autotune(rsr_ctx *ctx, const rsr_population *pop, rsr_dataset ds, const rsr_dataset *ds_per_program,
                         int reps, char *report, size_t report_len);

/* Number of this library's kernel launches issued on the context since
 * creation (device-side work the host enqueued). */
RSR_API uint64_t rsr_ctx_launch_count(rsr_ctx *ctx);
/* Bytes copied host->device and device->host by the last evaluation call. */
RSR_API int rsr_ctx_last_transfer(rsr_ctx *ctx, uint64_t *h2d_bytes, uint64_t *d2h_bytes);
/* Write bytes of zeros over a device scratch buffer larger than L2. */
RSR_API int rsr_flush_l2(rsr_ctx *ctx);
RSR_API int rsr_synchronize(rsr_ctx *ctx);
/* Measured FP32 throughput of this device in unfused lane-operations per
 * second (independent multiply and add chains): the roofline denominator of
 * the interpreter kernels. */
RSR_API int rsr_measure_fp32_peak(rsr_ctx *ctx, double *lane_ops_per_s);

/* ------------------------------------------------------ host encoder */
/* Validation against a feature count (0 = skip feature-range checks); does
 * not touch the device.  Returns RSR_OK or RSR_EPROGRAM. */
RSR_API int rsr_validate_program(const rsr_program *prog, uint32_t num_features);
/* Analysis summary used by the tests: max depth per typed stack
 * (F, V2, V3, M2, M3) in the reference's own evaluation order and after
 * reordering, and whether the register-stack kernel accepts the program. */
typedef struct rsr_program_info {
    uint32_t depth_ref[5];
    uint32_t depth_fast[5];
    uint32_t n_uops_fast;
    uint32_t n_uops_plain;
    int32_t fast_profile;        /* -1 when only the slot-file kernel applies */
    uint32_t flops_per_point;    /* algorithmic FP32 lane-ops incl. the MSE epilogue */
} rsr_program_info;
RSR_API int rsr_program_analyze(const rsr_program *prog, uint32_t num_features, rsr_program_info *info);
/* Device encoding of a program, for diagnostics and tests: form 0 = slot
 * form (3 words per instruction), 1 = accumulator form (one word per
 * micro-op), 2 = tape form (adjoint), 3 = slot form followed by its slot
 * count and flags (1: stack_f[0] never written, 2: slots need zeroing),
 * 4 = the same three from rsr_compute_mse_noalloc's fixed-array encoder
 * (RSR_EINVAL beyond its limits), 5 = the register adjoint's code preceded
 * by its kernel profile (0xFFFFFFFF: none), tape slots and five stack
 * depths.  Writes up to cap words and the full length to *len. */
RSR_API int rsr_program_encoding(const rsr_program *prog, uint32_t num_features, int form, uint32_t *out,
                                 uint32_t cap, uint32_t *len);

#ifdef __cplusplus
}
#endif
#endif /* RSR_GPU_H */
