/*
 * tbr.h -- C ABI of the B200 absolute-pose RANSAC engine (libtbr.so).
 *
 * Plain pointers, sizes and status codes only; no C++ or framework types.
 * The C++ drop-in shim in include/TbrCudaPnP/ (namespace TbrCudaPnP) and the
 * Python package turboransac_b200 are both thin layers over these calls.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   estimate_absolute_pose_cuda  Module/TbrCudaPnP/include/TbrCudaPnP/entry.h:13-19
 *                                (src/entry.cu:28-144)      -> tbr_estimate_absolute_pose
 *   get_inliers_mx               entry.h:22-25 (entry.cu:12-26) -> tbr_get_inliers
 *   bundle_adjust_cuda           include/TbrCudaPnP/ba.cuh:17-24 (src/ba.cu:111-130)
 *                                                            -> tbr_bundle_adjust
 *   turbo_ransac_pnp             include/TbrCudaPnP/turbo_ransac.cuh:13-19 (internal; its
 *                                per-round host loop src/turbo_ransac.cu:151-259 becomes the
 *                                device-side step engine behind all calls below)
 *   RansacOptions_cuda / RansacStats_cuda / BundleOptions_cuda / BundleStats_cuda
 *                                include/TbrCudaPnP/utils.h:14-72 -> tbr_*_options, tbr_stats
 *   the evaluator's per-frame loop TbrMain/src/main.cu:241-259 -> tbr_estimate_batch,
 *                                tbr_server_* (no reference counterpart beyond that loop)
 *
 * Error behaviour: the reference's CHECK macro prints and calls exit()
 * (include/TbrCudaPnP/cudaCheck.h:4-14); every call here instead returns a
 * tbr_status and leaves the process running. tbr_last_error() gives a message.
 *
 * Threading: a tbr_context owns one CUDA stream and its device workspace; use
 * one context per host thread. Calls on one context are synchronous unless
 * documented otherwise.
 */
#ifndef TBR_H
#define TBR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TBR_ABI_VERSION 1

typedef enum tbr_status {
    TBR_OK = 0,
    TBR_ERR_INVALID_ARG = 1, /* n < 3, size mismatch, bad pointer or option */
    TBR_ERR_OOM = 2,         /* device workspace or budget exhausted */
    TBR_ERR_CUDA = 3,        /* a CUDA runtime call failed */
    TBR_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
    TBR_ERR_CANCELLED = 5,   /* request cancelled by the caller */
    TBR_ERR_NOT_READY = 6,   /* server: nothing completed yet */
    TBR_ERR_CAPACITY = 7,    /* server: admission refused (queue full) */
    TBR_ERR_INTERNAL = 8
} tbr_status;

/* Mirrors RansacOptions_cuda (utils.h:14-31), field for field. */
typedef struct tbr_ransac_options {
    uint64_t max_iterations;      /* reference meaning: samples per round (the CUDA grid size) */
    uint64_t min_iterations;
    double dyn_num_trials_mult;
    double success_prob;
    double max_reproj_error;      /* pixels */
    double max_epipolar_error;
    uint64_t seed;
    int32_t progressive_sampling;
    uint64_t max_prosac_iterations;
    int32_t real_focal_check;
    int32_t score_initial_model;
} tbr_ransac_options;

/* Mirrors BundleOptions_cuda (utils.h:42-58). loss_type: 0 TRIVIAL, 1 TRUNCATED,
 * 2 HUBER, 3 CAUCHY, 4 TRUNCATED_LE_ZACH. */
typedef struct tbr_bundle_options {
    uint64_t max_iterations;
    int32_t loss_type;
    double loss_scale;
    double gradient_tol;
    double step_tol;
    double initial_lambda;
    double min_lambda;
    double max_lambda;
    int32_t verbose;
} tbr_bundle_options;

/* Extensions with no reference field. Zero-initialised = reference behaviour. */
typedef struct tbr_ext_options {
    /* 0 (default): the reference's hard-coded choices -- success_prob 0.9999,
     * trials multiplier 3, 100000-sample cap, default BundleOptions with a
     * 1/f loss scale (turbo_ransac.cu:145,227,231; entry.cu:122-123).
     * 1: honour success_prob, dyn_num_trials_mult, min_iterations,
     * progressive_sampling / max_prosac_iterations (PROSAC over points sorted
     * by decreasing quality) and the caller's bundle options; in
     * tbr_bundle_adjust also the loss type
     * (TRIVIAL, TRUNCATED, HUBER, CAUCHY) and the per-point weights, which
     * the reference ignores (ba.cu:111-130). */
    int32_t honor_options;
    int32_t skip_refine;          /* 1: return the RANSAC pose, no LM */
    int64_t force_samples;        /* > 0: score exactly this many samples, no early stop */
    int64_t max_total_samples;    /* 0 = 100000 */
    uint64_t seed;                /* Philox key of the sampler (0 = ransac.seed) */
    const int32_t *replay_idx;    /* host: replayed triples, replay_count*3 int32 */
    int64_t replay_count;
    int32_t hyp_per_thread;       /* scoring tile: 0 = default (the tensor-core kernel), else 2, 4, 6
                                     or 8 hypotheses per lane of the FP32 kernel */
    int32_t chunk_points;         /* scoring tile: 0 = auto, else points per work item */
    /* Stop rule K = ceil(3 log(1-p) / log(1-w^3)) beyond the int range: the
     * reference's double->int assignment (turbo_ransac.cu:231) is undefined
     * there and x86 yields INT_MIN, ending the loop after one round.
     * 0 (default): saturate -- keep sampling up to the cap; 1: reproduce x86. */
    int32_t stop_rule_x86_quirk;
    int32_t points_per_iter;      /* scoring tile: 0 = default, 2 or 4 points per inner step of the
                                     FP32 kernel (an FP32 field alone selects the FP32 kernel, the
                                     other field then 4 / 2), 128 = tensor-core scoring (tcgen05 MMA
                                     over 128-point tiles, 32 hypotheses per block; the default) */
} tbr_ext_options;

/* Results of one estimate. The reference returns RansacStats_cuda unfilled except
 * model_score = 0 (entry.cu:69,141); these are filled. */
typedef struct tbr_stats {
    int64_t samples;              /* minimal samples drawn */
    int64_t rounds;
    int64_t hypotheses;           /* P3P solutions scored */
    int64_t ransac_inliers;       /* FP64 inlier count of the RANSAC best (selection pass) */
    int64_t num_inliers;          /* inliers of the pre-LM pose (entry.cu:83 semantics) */
    double inlier_ratio;          /* num_inliers / n */
    double model_score;           /* FP64 MSAC score of the RANSAC best (normalized units) */
    int64_t best_sample;          /* sample id of the best hypothesis, -1 if none */
    int32_t best_solution;
    int32_t steps;                /* engine steps used */
    int64_t candidates_rescored;  /* hypotheses re-ranked in FP64 */
    int32_t candidate_overflow;   /* 1 if a single round had more FP64 re-rank candidates than
                                     fit (4096; possible only with more than 1024 samples per
                                     round) and one inside the FP32 error band was dropped: the
                                     selection may then differ from the FP64 pipeline's */
    int32_t lm_iterations;
    int32_t lm_invalid_steps;
    double lm_initial_cost;
    double lm_cost;
    double gpu_ms;                /* device time of the call (CUDA events) */
} tbr_stats;

typedef struct tbr_context tbr_context;

/* Returns TBR_ABI_VERSION. */
int tbr_abi_version(void);
/* Thread-local message of the last failing call on this thread. */
const char *tbr_last_error(void);

/* Fills *opts with the reference's defaults (utils.h:14-31 / :42-58). */
void tbr_default_ransac_options(tbr_ransac_options *opts);
void tbr_default_bundle_options(tbr_bundle_options *opts);

/* device: CUDA ordinal. workspace_bytes: device memory the context may use
 * (0 = 1 GiB). The workspace is allocated once and reused by every call. */
tbr_status tbr_context_create(int device, uint64_t workspace_bytes, tbr_context **out);
/* Also frees every batch made on the context that is still alive (a batch
 * uses the context's workspace and stream): those handles are dead afterwards,
 * and tbr_batch_destroy on one is a no-op, any other call on one returns
 * TBR_ERR_INVALID_ARG. Uncollected tickets (tbr_estimate_batch_submit) are
 * freed the same way: collect on one returns TBR_ERR_INVALID_ARG. A server
 * takes only the device from its context and may outlive it. */
void tbr_context_destroy(tbr_context *ctx);

/* estimate_absolute_pose_cuda (entry.h:13-19). Host buffers:
 *   points2D n*2 pixels (float64), points3D n*3 (float64), K = (fx, fy, cx, cy).
 * Outputs: q (w, x, y, z), t (X_cam = R X + t), inliers (n bytes, may be NULL),
 * stats (may be NULL). ext may be NULL. */
tbr_status tbr_estimate_absolute_pose(tbr_context *ctx, const double *points2D,
                                      const double *points3D, int64_t n, const double K[4],
                                      int32_t width, int32_t height,
                                      const tbr_ransac_options *ransac_opt,
                                      const tbr_bundle_options *bundle_opt,
                                      const tbr_ext_options *ext, double q[4], double t[3],
                                      uint8_t *inliers, tbr_stats *stats);

/* get_inliers_mx (entry.h:22-25): x n*2 normalized coordinates, X n*3,
 * pose (q, t); inlier iff squared reprojection error < sq_threshold and
 * depth > 0. Runs on the device; returns the count in *count (may be NULL). */
tbr_status tbr_get_inliers(tbr_context *ctx, const double q[4], const double t[3],
                           const double *x, const double *X, int64_t n, double sq_threshold,
                           uint8_t *inliers, int64_t *count);

/* bundle_adjust_cuda (ba.cuh:17-24): LM refinement of (q, t) in place on n
 * correspondences x (n*2, image units of the camera), X (n*3) with camera
 * K = (fx, fy, cx, cy). weights (n) may be NULL; as in the reference the
 * weights and loss_type are ignored unless ext->honor_options is set, and
 * the loss is Cauchy with scale opt->loss_scale. */
tbr_status tbr_bundle_adjust(tbr_context *ctx, const double *x, const double *X, int64_t n,
                             const double K[4], double q[4], double t[3],
                             const tbr_bundle_options *opt, const double *weights,
                             const tbr_ext_options *ext, tbr_stats *stats);

/* ---------------------------------------------------------------- batch --
 * Many frames of uneven size in one persistent, CUDA-graph-captured launch
 * sequence. A frame is described by host pointers; the call copies them in,
 * runs every frame to completion and copies results out. Every batched entry
 * point (here, the batch object and the server) refuses with
 * TBR_ERR_INVALID_ARG what the plain call refuses: max_iterations < 1,
 * max_reproj_error <= 0 in the options, and a frame with n < 3, a NULL array
 * or a focal length <= 0. */
typedef struct tbr_frame_desc {
    const double *points2D;   /* n*2 pixels */
    const double *points3D;   /* n*3 */
    int64_t n;
    double K[4];
    uint64_t seed;            /* per-frame Philox key */
    double max_reproj_error;  /* pixels; <= 0: take ransac_opt->max_reproj_error */
} tbr_frame_desc;

typedef struct tbr_frame_result {
    double q[4];
    double t[3];
    tbr_status status;
    int32_t pad;
    tbr_stats stats;
} tbr_frame_result;

tbr_status tbr_estimate_batch(tbr_context *ctx, const tbr_frame_desc *frames, int32_t n_frames,
                              const tbr_ransac_options *ransac_opt,
                              const tbr_ext_options *ext, tbr_frame_result *results,
                              uint8_t *const *inliers /* n_frames pointers, NULL entries ok */);

/* Correspondences already in device memory (no reference counterpart): as
 * tbr_estimate_batch, but each frame's points2D / points3D are device pointers
 * on the context's GPU -- e.g. a GPU feature matcher's output -- and are copied
 * device-to-device into the workspace, with no host staging. When stream (a
 * cudaStream_t) is not NULL the copy waits for the work queued on it so far;
 * with NULL the caller guarantees the data is ready. Results and inlier masks
 * are written to host memory. */
tbr_status tbr_estimate_batch_device(tbr_context *ctx, const tbr_frame_desc *frames, int32_t n_frames,
                                     const tbr_ransac_options *ransac_opt, const tbr_ext_options *ext,
                                     void *stream, tbr_frame_result *results, uint8_t *const *inliers);

/* Submitted batches (no reference counterpart; the reference's call,
 * estimate_absolute_pose_cuda in entry.h:13-19, returns only when its frame is
 * done): tbr_estimate_batch split into a submit that queues the whole run and
 * returns, and a collect that waits for it and writes the results. While the
 * device runs one batch the caller can prepare and submit the next, so the
 * host work of a call (descriptors, staging, launches, the result round
 * trip) overlaps the previous batch's device work.
 *   - Same frames, options, checks and results as tbr_estimate_batch (every
 *     frame's result is independent of the batch it runs in); at most 1024
 *     frames per submission.
 *   - The frames' arrays are read while the batch runs: they must stay valid
 *     and unchanged until tbr_estimate_batch_collect returns for the ticket.
 *   - A context has two sets of call buffers. Two submitted batches can have
 *     device work queued at once; submitting a third first waits for the
 *     oldest one's device work (its results stay with its ticket).
 *   - The frames hold their workspace until collected: a submission that does
 *     not fit beside the uncollected ones fails with TBR_ERR_OOM (points) or
 *     TBR_ERR_CAPACITY (frame slots).
 *   - Every other call on the context first waits for the device work of all
 *     submitted batches (their results stay with their tickets).
 *   - collect(ticket, results, inliers): results may be NULL (the ticket is
 *     released without results); inliers as in tbr_estimate_batch. The ticket
 *     is freed by collect, whatever it returns, and by tbr_context_destroy. */
typedef struct tbr_ticket tbr_ticket;
tbr_status tbr_estimate_batch_submit(tbr_context *ctx, const tbr_frame_desc *frames, int32_t n_frames,
                                     const tbr_ransac_options *ransac_opt, const tbr_ext_options *ext,
                                     tbr_ticket **ticket);
tbr_status tbr_estimate_batch_collect(tbr_ticket *ticket, tbr_frame_result *results, uint8_t *const *inliers);
/* The submitted form of tbr_estimate_batch_device (same rules as above, same
 * collect): the frames' arrays are device memory of the context's GPU, copied
 * after the work queued so far on `stream` (a cudaStream_t; NULL: the caller
 * guarantees the data is ready), and must stay unchanged until collect. */
tbr_status tbr_estimate_batch_device_submit(tbr_context *ctx, const tbr_frame_desc *frames, int32_t n_frames,
                                            const tbr_ransac_options *ransac_opt, const tbr_ext_options *ext,
                                            void *stream, tbr_ticket **ticket);

/* Device-resident batch: upload once (host->device), run many times with the
 * inputs already in HBM, download results. run() launches the captured graph
 * on the context stream; it is what the throughput measurement times. */
typedef struct tbr_batch tbr_batch;
tbr_status tbr_batch_create(tbr_context *ctx, const tbr_frame_desc *frames, int32_t n_frames,
                            const tbr_ransac_options *ransac_opt, const tbr_ext_options *ext,
                            tbr_batch **out);
tbr_status tbr_batch_run(tbr_batch *b);      /* asynchronous on the context stream */
tbr_status tbr_batch_sync(tbr_batch *b);     /* waits; returns the first device error */
tbr_status tbr_batch_results(tbr_batch *b, tbr_frame_result *results);
void tbr_batch_destroy(tbr_batch *b);        /* no-op if its context already freed it */

/* Per-kernel device time of one batch run, stepped from the host with a CUDA
 * event pair around every kernel launch on the context stream (slower than
 * tbr_batch_run; for measurement only). pairs_scored = hypothesis x point
 * pairs evaluated by the FP32 scoring kernel. */
typedef struct tbr_kernel_profile {
    char name[32];
    double total_ms;
    int64_t launches;
} tbr_kernel_profile;
tbr_status tbr_batch_profile(tbr_batch *b, tbr_kernel_profile *out, int32_t max, int32_t *n_out,
                             uint64_t *pairs_scored);

/* Scoring-shape autotuner (no reference counterpart). Times the batch's graph
 * `repeats` times under each candidate shape -- FP32: hypotheses per warp block
 * (32 x hyp_per_thread: 64, 128, 192, 256), points per iteration (2, 4) and points
 * per work-item tile (0 = sized from the step's work, 256, 512, 1024, 2048);
 * tensor cores: points_per_iter = 128 (32 hypotheses per block, reported as
 * hyp_per_thread = 1) with tiles 0 and 8192; 32 candidates in all --
 * and keeps the fastest for later tbr_batch_run calls. The shape changes only
 * the order of FP32 partial sums inside the filter; every candidate within the
 * filter band is re-scored in FP64, so results do not depend on it. entries
 * (may be NULL) receive up to max candidates with their mean device ms. */
typedef struct tbr_tune_entry {
    int32_t hyp_per_thread;
    int32_t points_per_iter;
    int32_t chunk_points;
    int32_t pad;
    double ms;
} tbr_tune_entry;
tbr_status tbr_batch_autotune(tbr_batch *b, int32_t repeats, tbr_tune_entry *entries, int32_t max,
                              int32_t *n_out, tbr_tune_entry *best);

/* Measured FP32 FMA throughput of the context's device (packed FP32x2 FMA
 * chains on every SM, CUDA-event timed): the denominator of the scoring
 * kernel's roofline. */
tbr_status tbr_measure_fp32_peak(tbr_context *ctx, double *tflops);

/* -------------------------------------------------------------- serving --
 * Continuous batching: a worker thread advances every admitted frame by one
 * engine step at a time; requests that arrive while others run are admitted
 * into free slots as memory frees up, so their work overlaps on the device. */
typedef struct tbr_server tbr_server;
typedef struct tbr_server_config {
    uint64_t workspace_budget_bytes;  /* device bytes for admitted frames' state */
    int32_t max_slots;                /* frames resident at once */
    int32_t max_queue;                /* pending requests before submit refuses */
    tbr_ransac_options ransac;
    tbr_ext_options ext;
} tbr_server_config;

typedef struct tbr_server_result {
    uint64_t request_id;
    tbr_status status;
    int32_t pad;
    double q[4];
    double t[3];
    tbr_stats stats;
    double submit_to_done_ms;         /* host wall clock from submit to completion */
} tbr_server_result;

/* Counters of the request loop since creation. The loop overlaps staging of
 * new requests (host copies into pinned memory) with the step running on the
 * device; device_wait_ms is the time it waited for steps to finish. */
typedef struct tbr_server_stats {
    int64_t submitted, admitted, completed;
    int64_t steps;          /* engine steps launched */
    int64_t resident_sum;   /* sum over steps of resident frames (mean = /steps) */
    double host_stage_ms;   /* picking and copying admissions */
    double device_wait_ms;  /* waiting for the step in flight */
    double host_retire_ms;  /* downloading and publishing results */
    double host_launch_ms;  /* uploads and step launches */
    int64_t pairs_scored;   /* (hypothesis, point) pairs scored by the steps retired so far */
} tbr_server_stats;

tbr_status tbr_server_create(tbr_context *ctx, const tbr_server_config *cfg, tbr_server **out);
/* Copies the frame's host arrays; returns immediately. */
tbr_status tbr_server_submit(tbr_server *s, const tbr_frame_desc *frame, uint64_t *request_id);
/* Does not copy: the frame's arrays are read when the request is admitted, so
 * they must stay valid and unchanged until its result has been polled. */
tbr_status tbr_server_submit_nocopy(tbr_server *s, const tbr_frame_desc *frame, uint64_t *request_id);
tbr_status tbr_server_get_stats(tbr_server *s, tbr_server_stats *out);
/* Moves up to max completed results into out; *n_out = number written. */
tbr_status tbr_server_poll(tbr_server *s, tbr_server_result *out, int32_t max, int32_t *n_out);
tbr_status tbr_server_cancel(tbr_server *s, uint64_t request_id);
/* Blocks until every submitted request has completed or failed. */
tbr_status tbr_server_drain(tbr_server *s);
void tbr_server_destroy(tbr_server *s);

/* ------------------------------------------------------------ diagnostics --
 * Score replayed samples exactly as one engine step does and return, per
 * hypothesis (in sample order, solution order): id = sample*4 + solution, the
 * FP64 P3P pose (12 doubles, [R | t] row-major), the FP32 MSAC score in units
 * of tau^2 and, when counts != NULL, the inlier count decided in FP32 with an
 * FP64 recheck of pairs near the threshold. Returns the number of hypotheses
 * in *n_hyp (capped at cap). Used by the parity tests. */
tbr_status tbr_debug_score_samples(tbr_context *ctx, const double *points2D,
                                   const double *points3D, int64_t n, const double K[4],
                                   double max_reproj_error, const int32_t *triples,
                                   int64_t n_samples, int64_t *ids, double *poses,
                                   float *scores32, int64_t *counts, int64_t cap,
                                   int64_t *n_hyp, const tbr_ext_options *ext);

/* Failure-path check (no reference counterpart): one kernel waits on an
 * mbarrier that nothing completes, giving up after `polls` tries (1 .. 2^22)
 * as every wait of the engine's kernels does after its own limit. Returns
 * TBR_ERR_TIMEOUT, read from the device's error word like any expired wait;
 * the context stays usable. Used by the tests. */
tbr_status tbr_debug_bounded_wait(tbr_context *ctx, uint32_t polls);

/* --------------------------------------------------------- no allocation --
 * No counterpart in the reference. FP64 truncated-MSAC scores and inlier counts
 * of n_poses poses (n_poses*12 doubles, [R | t] row-major) over n device-resident
 * correspondences x_dev (n*2 normalized coordinates) and X_dev (n*3), written to
 * scores_dev[n_poses] and counts_dev[n_poses], asynchronously on `stream`
 * (a cudaStream_t; NULL = the legacy default stream).
 * For callers that must not allocate device memory -- code running inside
 * another runtime's memory pool or an allocation-free real-time loop: this
 * call performs no cudaMalloc or other allocation. Its working memory is one
 * fixed array of about 400 KB compiled into the library, which every GPU that
 * loads the library keeps until the process exits. Limits and rules:
 *  - at most 1024 poses per call (larger requests fail with TBR_ERR_INVALID_ARG);
 *    sq_threshold must be positive and finite (else TBR_ERR_INVALID_ARG);
 *  - the device of `stream` must be the current device (else TBR_ERR_INVALID_ARG);
 *  - the first call on each device looks up the array's device address (with
 *    that device current), so make that first call before any stream capture;
 *    the address is kept for the life of the process, so after a
 *    cudaDeviceReset (which unloads the library's device code) the call must
 *    not be used again on that device;
 *  - all calls share the array: calls that overlap on the GPU (different
 *    streams, or other threads) race -- order them on one stream or with events. */
tbr_status tbr_msac_score_noalloc(const double *x_dev, const double *X_dev, int64_t n,
                                  const double *poses_dev, int32_t n_poses, double sq_threshold,
                                  double *scores_dev, int64_t *counts_dev, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TBR_H */
