/*
 * FP64 CPU oracle for the absolute-pose RANSAC path (TEST INFRASTRUCTURE).
 *
 * This is a plain-C++ restatement of the reference's algorithm, used only as
 * the checker by tests/, by __graft_entry__.smoke() and by the CPU-baseline
 * leg of bench.py. The product path (turboransac_b200, libtbr.so) never links
 * or calls it.
 *
 * Parity pin: the P3P solver, the pose/quaternion helpers, the Cauchy loss and
 * the 6x6 Cholesky are checked bit-for-bit / to 1e-12 against the reference's
 * own header code compiled on the host (oracle/ref_harness.cpp, built into
 * oracle/_ref by oracle/Makefile), and against the committed fixtures in
 * tests/golden/ that the same harness generated.
 *
 * Pose convention (all functions): P is 3x4 row-major, P[r*4+c], X_cam = R*X + t,
 * i.e. the first three rows of the reference's 4x4 row-major pose buffer.
 */
#ifndef TBR_ORACLE_H
#define TBR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Philox4x32-10 (Salmon et al., SC'11), the counter-based generator the GPU
 * sampler uses. ctr[4], key[2] -> out[4]. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Draw `count` ordered triples of distinct indices in [0,n) for sample ids
 * first_sample .. first_sample+count-1 of the stream keyed by `seed`.
 * idx_out has count*3 entries. Same arithmetic as the device sampler. */
void orc_sample_triples(uint64_t seed, int64_t first_sample, int64_t count, int64_t n,
                        int32_t *idx_out);

/* Lambda-Twist-type P3P following p3p.cuh:9-222. x: 3 unit bearings (row i =
 * bearing i), X: 3 world points (row i). Writes up to 4 poses of 12 doubles to
 * poses_out and returns their number. */
int orc_p3p(const double *x, const double *X, double *poses_out);

/* Bearing of a normalized image point: (x, y, 1) / ||(x, y, 1)||
 * (ransac.cuh:196-200). */
void orc_bearing(double x, double y, double out[3]);

/* Truncated MSAC score of one pose over n points (msac.cuh:18-56 and the
 * block sum ransac.cuh:259-335): score = sum_{inliers} r^2 + (n - count) * sq_thr. */
void orc_msac(const double *xn, const double *X, int64_t n, const double *P, double sq_thr,
              double *score, int64_t *count);

/* Quaternion helpers (pose_utils.cuh). q = (w, x, y, z). R row-major 3x3. */
void orc_rotmat_to_quat(const double *R, double q[4]);
void orc_quat_to_rotmat(const double q[4], double *R);

/* get_inliers_mx (entry.cu:12-26): inlier iff ||hnormalized(R X + t) - x||^2 < sq_thr
 * and depth > 0. R is built from q via quat_to_rotmat as CameraPose_cuda::R() does. */
int64_t orc_get_inliers(const double q[4], const double t[3], const double *xn, const double *X,
                        int64_t n, double sq_thr, uint8_t *inliers);

typedef struct orc_ransac_cfg {
    int64_t samples_per_round;  /* B = RansacOptions_cuda::max_iterations */
    int64_t max_total_samples;  /* reference hard-codes 100000 (turbo_ransac.cu:145) */
    double success_prob;        /* reference hard-codes 0.9999 (turbo_ransac.cu:227) */
    double trials_mult;         /* reference hard-codes 3 (turbo_ransac.cu:231) */
    int64_t force_samples;      /* > 0: score exactly this many samples, no early stop */
    uint64_t seed;              /* Philox key */
    const int32_t *replay;      /* optional replayed triples (count*3) */
    int64_t replay_count;
    int threads;                /* worker threads over samples (>=1) */
    int quirk;                  /* 1: stop rule with the x86 int-conversion result (INT_MIN) */
    int64_t min_samples;        /* no stop before this many samples (0: none) */
    int32_t prosac;             /* 1: PROSAC sampling over points sorted by quality */
    double prosac_TN;           /* T_N: samples after which PROSAC draws uniformly */
} orc_ransac_cfg;

/* PROSAC growth table (Chum & Matas, CVPR 2005): Tp[k-3] = T'_k for k = 3..n,
 * T'_3 = 1, T'_{k+1} = T'_k + ceil(T_{k+1} - T_k), T_k = T_N * C(k,3) / C(n,3)
 * evaluated as ((T_N * (k/n)) * ((k-1)/(n-1))) * ((k-2)/(n-2)). n-2 entries. */
void orc_prosac_table(int64_t n, double TN, int64_t *Tp);

/* PROSAC ordered triple of sample `sample` (0-based; iteration t = sample+1):
 * with g = #{k in 3..n-1 : T'_k <= t} and m = 3 + g, the triple is two
 * distinct indices of the first m-1 points and point m-1; once m = n and
 * T'_n < t it is the uniform triple of orc_sample_triples. */
void orc_prosac_triple(uint64_t seed, int64_t sample, int64_t n, const int64_t *Tp, int32_t out[3]);

typedef struct orc_ransac_out {
    double P[12];          /* best pose, identity if none */
    double score;          /* FP64 MSAC score of the best (DBL_MAX if none) */
    int64_t count;         /* its inlier count */
    int64_t best_sample;   /* sample id of the best (-1 if none) */
    int32_t best_sol;      /* P3P solution index within that sample */
    int32_t found;
    int64_t samples;       /* samples drawn */
    int64_t rounds;
    int64_t hypotheses;    /* P3P solutions scored */
} orc_ransac_out;

/* RANSAC with the reference's selection and adaptive-termination semantics
 * (turbo_ransac.cu:143-259, ransac.cuh:140-360). Optional per-hypothesis dump
 * (in sample order, solution order): scores, counts, (sample_id*4+sol) ids and
 * poses; hyp_cap bounds the dump. Returns 0 on success. */
int orc_ransac(const double *xn, const double *X, int64_t n, double sq_thr,
               const orc_ransac_cfg *cfg, orc_ransac_out *out,
               double *hyp_scores, int64_t *hyp_counts, int64_t *hyp_ids, double *hyp_poses,
               int64_t hyp_cap);

typedef struct orc_lm_opts {
    int64_t max_iterations;
    double loss_scale, gradient_tol, step_tol, initial_lambda, min_lambda, max_lambda;
    /* Honoured-options extension (the reference always uses Cauchy and unit
     * weights): 0 Cauchy, 1 truncated (robust_loss.cuh:10-22), 2 Huber,
     * 3 trivial; weights: NULL or one multiplier per point on loss and weight. */
    int32_t loss;
    const double *weights;
} orc_lm_opts;

typedef struct orc_lm_stats {
    int64_t iterations, invalid_steps;
    double initial_cost, cost, lambda, step_norm, grad_norm;
} orc_lm_stats;

/* One-frame Levenberg-Marquardt with the Cauchy loss (lm.cuh:15-171,
 * jaco.cuh:31-299, lm_utils.cuh:14-100). x: n*2 observations, X: n*3,
 * cam = (fx, fy, cx, cy). q, t are refined in place. */
void orc_lm(const double *x, const double *X, int64_t n, const double cam[4], double q[4],
            double t[3], const orc_lm_opts *opt, orc_lm_stats *stats);

typedef struct orc_estimate_info {
    orc_ransac_out ransac;
    orc_lm_stats lm;
    int64_t num_inliers;   /* inliers of the pre-LM pose (entry.cu:83) */
} orc_estimate_info;

/* The whole estimate_absolute_pose_cuda path (entry.cu:28-144): unproject,
 * RANSAC, inliers with the pre-LM pose, LM on the inliers in pixel/f units,
 * output (q, t). uv: n*2 pixels, X: n*3, K = (fx, fy, cx, cy). */
int orc_estimate(const double *uv, const double *X, int64_t n, const double K[4],
                 double max_reproj_error, const orc_ransac_cfg *cfg, int skip_refine,
                 double q[4], double t[3], uint8_t *inliers, orc_estimate_info *info);

/* Many frames at once, `threads` workers over frames (each frame single-threaded).
 * Arrays are concatenated; offsets[f] is the first point of frame f (n_frames+1
 * entries). seeds[f] keys frame f. q_out/t_out: n_frames*4 / n_frames*3. */
int orc_estimate_batch(const double *uv, const double *X, const int64_t *offsets,
                       const double *K, const uint64_t *seeds, int n_frames,
                       double max_reproj_error, int64_t samples_per_round, int threads,
                       double *q_out, double *t_out, int64_t *samples_out);

#ifdef __cplusplus
}
#endif

#endif
