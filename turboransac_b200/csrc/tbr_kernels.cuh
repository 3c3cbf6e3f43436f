// Kernels of one engine step (sm_100a). Host orchestration lives in tbr_engine.cu.
//
// A step advances every resident frame in the RANSAC state by a planned number
// of rounds:
//   k_plan          rounds to run this step per frame (adaptive-termination aware)
//   k_sample_p3p    one thread per minimal sample: Philox triple (or replay), FP64 P3P
//   k_score_plan    work items (frame, 32*HR hypotheses, point chunk)
//   k_score         FP32 truncated-MSAC filter pass (the hot kernel)
//   k_select        candidates within a safe band of each round's running minimum
//   k_rescore_plan / k_rescore   exact FP64 MSAC of the candidates (reference formula)
//   k_finalize      the reference's selection and stop rule, round by round
// then, for frames whose RANSAC ended:
//   k_inliers       get_inliers_mx semantics + ordered compaction of the inliers
//   k_lm            Levenberg-Marquardt, FP32 compensated J^T J / J^T r, FP64 solve
#pragma once

#include <cfloat>
#include <climits>
#include <cooperative_groups.h>
#include <cstdint>

#include "tbr_device.cuh"

namespace tbr {

constexpr int kSub = 64;                          // points per FP32 staging block
// Depth floor of the FP32 filter: the reciprocal of any smaller depth is 2^100.
constexpr float kDepthFloor = 0x1p-100f;
constexpr int kRescoreGroup = 8;  // FP64 re-rank: candidates of a frame scored together per point chunk
constexpr int kBlockFloat2 = kSub * 5;            // float2 entries per block
constexpr uint32_t kBlockBytes = kBlockFloat2 * 8;  // 2560 B per block
constexpr int kMaxRoundsPerStep = 128;
constexpr int kMaxCandFrame = 4096;               // FP64 re-rank candidates per frame and step
constexpr int kMaxRChunks = 32;                   // FP64 rescoring point chunks per frame
constexpr int kMaxScoreChunks = 64;               // FP32 scoring point chunks per frame
constexpr int kMaxActive = 1024;                  // frames advanced by one step
constexpr uint32_t kMaxPolls = 1u << 26;          // bounded mbarrier waits (~seconds)
constexpr int kScoreWarps = 4;                    // warps per scoring CTA
constexpr int kLMThreads = 256;       // per CTA of a cluster LM (two CTAs per SM)
constexpr int kLMSmallThreads = 384;  // one CTA per frame: 12 warps, no register spills

// kLMReady: RANSAC finished in the step stamped in lm_epoch; k_inliers takes it
// one step later (so that in the captured loop it can run beside the next
// step's RANSAC kernels without racing them) and moves it to kLMPending.
// kPending: admitted, its correspondences still on the way; every step kernel
// skips it until k_activate moves it to kRansac (a frame's samples and results
// do not depend on the step it starts in).
enum FrameStatus : int32_t {
    kFree = 0,
    kRansac = 1,
    kLMPending = 2,
    kDone = 3,
    kFailed = 4,
    kLMReady = 5,
    kPending = 6
};

enum Counter : int {
    kCScoreNext = 0,
    kCScoreTotal,
    kCRescoreNext,
    kCRescoreTotal,
    kCSamplesTotal,
    kCError,
    kCStillRansac,
    kCLMPending,
    kCWorkPairs,
    kCCandNext,
    kCSteps,
    kCPairsTotal,
    kCNum
};

enum ErrorBits : unsigned long long { kErrTimeout = 1ull, kErrOverflow = 2ull };

struct FrameResult {
    double q[4];
    double t[3];
    int64_t samples, rounds, hypotheses, ransac_inliers, num_inliers;
    double model_score;
    int64_t best_sample;
    int32_t best_sol, steps;
    int64_t rescored;
    int32_t overflow, lm_iters, lm_invalid, status;
    double lm_cost0, lm_cost;
};

struct __align__(16) FrameDev {
    // ---- inputs, fixed at admission ----
    int64_t n;
    int64_t blk_off;  // first staging block; the frame's points start at blk_off * kSub
    int32_t n_blocks;
    int32_t status;
    uint64_t seed;
    const int32_t *replay;  // device triples or nullptr
    int64_t replay_count;
    double K[4];
    double focal, tau, sq_thr;
    double centre[3];
    unsigned long long bmin[3], bmax[3];
    int64_t B;
    int64_t max_total;
    int64_t min_samples;  // no stop before this many samples (honoured min_iterations; else 0)
    double prosac_TN;     // PROSAC: samples after which it draws uniformly
    int32_t prosac;       // 1: PROSAC sampling (honoured progressive_sampling), table in Pools::prosac64
    int32_t split;        // > 0: at most this many rounds (forced mode: samples) per step, set when a
                          // step's re-rank candidates did not fit (k_select); results do not change
    int64_t force_samples;
    double log_missing, trials_mult;
    int32_t skip_refine, hr;  // hr: hypotheses per lane in the scoring pass (2 * HP)
    int32_t quirk;            // stop rule: 1 = x86 int-conversion quirk of the reference
    int32_t redo;             // 1: this step's candidates did not fit; k_finalize discards the step
    int64_t lm_max_iter;
    double lm_cam[4];  // camera of the LM residual: K/f for the estimate path, K for bundle_adjust
    double lm_inv_sq_thr, lm_grad_tol, lm_step_tol, lm_lambda0, lm_min_lambda, lm_max_lambda;
    double lm_thr;            // loss scale (LM units) of the honoured truncated / Huber losses
    int32_t lm_loss;          // kLossCauchy (the reference's), kLossTruncated, kLossHuber, kLossTrivial
    int32_t lm_weighted;      // 1: per-point multipliers in Pools::lw64 (bundle adjust, honoured)
    int32_t chunk_points, max_rounds_step;  // max_rounds_step: 0 = kMaxRoundsPerStep
    // ---- RANSAC progress ----
    int64_t samples_done, rounds_done, hyps_done;
    int32_t steps, found;
    double best_score;
    int64_t best_count, best_sample;
    int32_t best_sol, overflow;
    double best_P[12];
    int64_t rescored;
    // ---- current step ----
    int64_t step_first, step_samples, step_rounds, step_div;
    int64_t hyp_base;
    int32_t hyp_count, n_hblocks;
    int32_t n_chunks, chunk_blocks;
    int64_t part_base, hb_base;
    int32_t cand_count, n_rchunks;
    int64_t rchunk, cand_base;
    unsigned long long round_min[kMaxRoundsPerStep];
    int32_t round_hyps[kMaxRoundsPerStep];
    // ---- LM ----
    int64_t num_inliers;
    int64_t lm_epoch;  // engine step in which RANSAC finished
    int32_t lm_force_cluster, pad9;  // bundle_adjust path: always the cluster LM
};

struct Pools {
    FrameDev *frames;
    FrameResult *results;
    const int32_t *active;  // slots advanced by this launch
    int32_t n_active;
    int32_t num_sms;
    int64_t lm_cluster_min;  // inliers from which a frame's LM runs on a CTA cluster
    // per point (blocks * kSub entries)
    const double *uv64;  // raw pixels (2/pt)
    const double *X64;   // world points (3/pt)
    double *xn64;        // normalized image points (2/pt)
    uint8_t *mask;       // final inlier mask (1/pt)
    double *lx64;        // LM: pixels / f (2/pt)
    double *lX64;        // LM: world points (3/pt)
    double *lw64;        // LM: per-point loss multipliers (bundle adjust with honoured weights)
    int64_t *prosac64;   // PROSAC growth table of a frame, one entry per point (T'_k at k - 3)
    float2 *pts32;       // staging blocks: [X|Y|Z|-x/tau|-y/tau] x kSub, each value duplicated
    // step prefixes (n_active + 1)
    int64_t *sample_prefix;
    int64_t *item_prefix;
    int64_t *ritem_prefix;
    // hypotheses
    double *hP64;
    float *hP32;
    int64_t *hId;
    float *hS32;
    float *part;
    unsigned *hb_arrive;
    int64_t max_hyps, max_parts, max_hb;
    // FP64 re-rank candidates: one pool shared by the step, a region per frame
    int64_t cand_cap;
    int32_t *cHyp;   // hypothesis index within the frame's step region
    double *cS64;
    int64_t *cCnt;
    double *cpS;     // candidate * kMaxRChunks + chunk
    int32_t *cpC;
    unsigned *c_arrive;
    unsigned long long *counters;
    // debug: per-hypothesis counts (tbr_debug_score_samples)
    int64_t *dbg_counts;
};

// ------------------------------------------------------------- helpers -----
// Samples the stop rule requires (turbo_ransac.cu:223-231):
//   K = ceil(log(1 - p) / log(1 - w^3) * mult),  w = best inlier count / n.
// The reference assigns K to an int; for K beyond the int range (w below about
// 0.0024, or no inlier at all) that conversion is undefined behaviour, which
// x86 resolves to INT_MIN and the round loop stops after its first round.
// quirk = 1 reproduces that; quirk = 0 (default) saturates, so a frame without
// a usable model keeps sampling up to the sample cap.
__device__ __forceinline__ int64_t needed_samples(int64_t inliers, int64_t n, double log_missing,
                                                  double mult, int quirk) {
    const double w = (double)inliers / (double)n;
    const double prob_outlier = 1.0 - pow(w, 3.0);
    const double v = ceil(log_missing / log(prob_outlier) * mult);
    if (quirk) {
        if (!(v >= -2147483648.0 && v < 2147483648.0)) return (int64_t)INT_MIN;
        return (int64_t)(int)v;
    }
    if (inliers <= 0 || !(v == v) || v >= 2147483647.0) return (int64_t)INT_MAX;
    if (v <= -2147483648.0) return (int64_t)INT_MIN;
    return (int64_t)v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide exclusive scan over blockDim.x <= 1024 values; returns the
// exclusive prefix, writes the total. Uses 33 int64 of shared scratch.
__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t *sh, int64_t &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int64_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) sh[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < nw ? sh[lane] : 0;
        int64_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t u = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += u;
        }
        if (lane < nw) sh[lane] = wi - w;
        if (lane == nw - 1) sh[32] = wi;
    }
    __syncthreads();
    const int64_t r = sh[warp] + incl - v;
    total = sh[32];
    __syncthreads();
    return r;
}

__device__ __forceinline__ int find_segment(const int64_t *prefix, int n, int64_t g) {
    int lo = 0, hi = n - 1;  // largest i with prefix[i] <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void flag_error(const Pools &P, unsigned long long bits) {
    atomicOr(&P.counters[kCError], bits);
}

// ----------------------------------------------------------- admission -----
// AABB of the frame's world points (ordered-integer atomics: order independent).
__global__ void k_prep_bounds(Pools P) {
    const int a = blockIdx.y;
    if (a >= P.n_active) return;
    FrameDev &f = P.frames[P.active[a]];
    const int64_t base = f.blk_off * kSub;
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < f.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double v0 = P.X64[3 * (base + i)], v1 = P.X64[3 * (base + i) + 1], v2 = P.X64[3 * (base + i) + 2];
        if (!(isfinite(v0) && isfinite(v1) && isfinite(v2))) continue;  // staged as an outlier
        const double v[3] = {v0, v1, v2};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = fmin(lo[k], v[k]);
            hi[k] = fmax(hi[k], v[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fmin(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
            hi[k] = fmax(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&f.bmin[k], dbl_to_ordered(lo[k]));
            atomicMax(&f.bmax[k], dbl_to_ordered(hi[k]));
        }
    }
}

// Normalized coordinates (Camera_cuda::unproject, camera.cuh:51-62) and the FP32
// staging blocks: centred world points and -x/tau, -y/tau, each duplicated so
// that one 64-bit lane pair feeds both halves of a packed FP32x2 instruction.
__global__ void k_prep_pack(Pools P) {
    const int a = blockIdx.y;
    if (a >= P.n_active) return;
    FrameDev &f = P.frames[P.active[a]];
    const int64_t base = f.blk_off * kSub;
    double cc[3];
    for (int k = 0; k < 3; ++k) {  // no finite point: centre 0
        cc[k] = 0.5 * (ordered_to_dbl(f.bmin[k]) + ordered_to_dbl(f.bmax[k]));
        if (!isfinite(cc[k])) cc[k] = 0.0;
    }
    const double c0 = cc[0], c1 = cc[1], c2 = cc[2];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        f.centre[0] = c0;
        f.centre[1] = c1;
        f.centre[2] = c2;
    }
    const double fx = f.K[0], fy = f.K[1], cx = f.K[2], cy = f.K[3];
    const double itau = 1.0 / f.tau;
    const int64_t npad = (int64_t)f.n_blocks * kSub;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npad;
         i += (int64_t)gridDim.x * blockDim.x) {
        float v[5];
        if (i < f.n) {
            const double u = P.uv64[2 * (base + i)], w = P.uv64[2 * (base + i) + 1];
            const double xn = (u - cx) / fx, yn = (w - cy) / fy;
            P.xn64[2 * (base + i)] = xn;
            P.xn64[2 * (base + i) + 1] = yn;
            v[0] = (float)(P.X64[3 * (base + i)] - c0);
            v[1] = (float)(P.X64[3 * (base + i) + 1] - c1);
            v[2] = (float)(P.X64[3 * (base + i) + 2] - c2);
            v[3] = (float)(-xn * itau);
            v[4] = (float)(-yn * itau);
            bool finite = true;
#pragma unroll
            for (int k = 0; k < 5; ++k) finite = finite && fabsf(v[k]) <= 0x1p80f;
            if (!finite) {  // non-finite (never an FP64 inlier) or beyond 2^80: outlier for every pose
                v[0] = v[1] = v[2] = 0.0f;
                v[3] = v[4] = 0x1p100f;
            }
        } else {
            v[0] = v[1] = v[2] = v[3] = v[4] = 0.0f;
        }
        float2 *blk = P.pts32 + (f.blk_off + i / kSub) * kBlockFloat2;
        const int j = (int)(i % kSub);
#pragma unroll
        for (int k = 0; k < 5; ++k) blk[k * kSub + j] = make_float2(v[k], v[k]);
    }
}

// PROSAC growth table of each PROSAC frame (one CTA per frame):
// T'_3 = 1, T'_{k+1} = T'_k + ceil(T_{k+1} - T_k), T_k = T_N C(k,3) / C(n,3)
// evaluated as ((T_N * (k/n)) * ((k-1)/(n-1))) * ((k-2)/(n-2)) with rounded
// operations only (no contraction), so the table is the oracle's bit for bit.
__device__ __forceinline__ double prosac_T(double TN, int64_t k, int64_t n) {
    const double a = __ddiv_rn((double)k, (double)n), b = __ddiv_rn((double)(k - 1), (double)(n - 1)),
                 c = __ddiv_rn((double)(k - 2), (double)(n - 2));
    return __dmul_rn(__dmul_rn(__dmul_rn(TN, a), b), c);
}
__global__ void __launch_bounds__(1024) k_prosac_table(Pools P) {
    __shared__ int64_t sh[33];
    const int a = blockIdx.x;
    if (a >= P.n_active) return;
    const FrameDev &f = P.frames[P.active[a]];
    if (!f.prosac) return;
    const int64_t n = f.n, cnt = n - 3;  // increments for k = 3 .. n-1
    int64_t *Tp = P.prosac64 + f.blk_off * kSub;
    const int64_t per = (cnt + blockDim.x - 1) / blockDim.x;
    const int64_t k0 = 3 + (int64_t)threadIdx.x * per, k1 = min(k0 + per, (int64_t)n);
    int64_t local = 0;
    for (int64_t k = k0; k < k1; ++k)
        local += (int64_t)ceil(__dsub_rn(prosac_T(f.prosac_TN, k + 1, n), prosac_T(f.prosac_TN, k, n)));
    int64_t tot;
    int64_t run = 1 + block_exclusive_scan(local, sh, tot);
    if (threadIdx.x == 0) Tp[0] = 1;
    for (int64_t k = k0; k < k1; ++k) {
        run += (int64_t)ceil(__dsub_rn(prosac_T(f.prosac_TN, k + 1, n), prosac_T(f.prosac_TN, k, n)));
        Tp[k - 2] = run;
    }
}

// ---------------------------------------------------------------- plan -----
// Rounds per frame for this step. The first step runs one round; later steps
// run exactly the rounds the current best's inlier ratio still requires under
// the reference's stop rule (turbo_ransac.cu:223-257), so a frame normally
// finishes in one or two steps while its samples, selection and stop point are
// those of the sequential round loop. Hypothesis-pool capacity is shared in
// frame order; a frame that does not fit waits for the next step.
__global__ void k_plan(Pools P) {
    __shared__ int64_t sh[33];
    const int a = threadIdx.x;
    int64_t samples = 0, rounds = 0, div = 0;
    FrameDev *f = nullptr;
    if (a < P.n_active) {
        f = &P.frames[P.active[a]];
        f->step_samples = 0;
        f->step_rounds = 0;
        f->hyp_count = 0;
        f->cand_count = 0;
        if (f->status == kRansac) {
            if (f->force_samples > 0) {
                samples = f->force_samples - f->samples_done;
                if (f->split > 0) samples = min(samples, (int64_t)f->split);
                rounds = 1;
                div = f->force_samples;
            } else {
                const int64_t max_rounds = (f->max_total + f->B - 1) / f->B;
                int64_t r = 1;
                if (f->rounds_done > 0) {
                    const int64_t need = needed_samples(f->found ? f->best_count : 0, f->n,
                                                        f->log_missing, f->trials_mult, f->quirk);
                    r = need / f->B + 1 - f->rounds_done;
                    if (need < 0 || r < 1) r = 1;
                }
                r = max(r, (f->min_samples + f->B - 1) / f->B - f->rounds_done);
                r = min(r, max_rounds - f->rounds_done);
                r = min(r, (int64_t)(f->max_rounds_step > 0 ? f->max_rounds_step : kMaxRoundsPerStep));
                // Growth cap: the frame's s-th step runs at most 4 * 2^(s-1) rounds,
                // so a stop bound that shrinks once a better model turns up wastes
                // at most the last step's overshoot.
                if (f->steps >= 1) r = min(r, (int64_t)4 << min(f->steps - 1, 5));
                if (f->split > 0) r = min(r, (int64_t)f->split);
                if (r < 1) r = 1;
                rounds = r;
                samples = r * f->B;
                div = f->B;
            }
        }
    }
    // Capacity: 4 hypotheses per sample at most.
    int64_t total;
    int64_t excl = block_exclusive_scan(4 * samples, sh, total);
    if (f && samples > 0 && excl + 4 * samples > P.max_hyps) {
        const int64_t room = P.max_hyps - excl;
        if (room <= 0) {
            samples = rounds = 0;
        } else if (f->force_samples > 0) {
            samples = room / 4;
        } else {
            rounds = room / (4 * f->B);
            samples = rounds * f->B;
        }
    }
    const int64_t hyp_excl = block_exclusive_scan(4 * samples, sh, total);
    const int64_t s_excl = block_exclusive_scan(samples, sh, total);
    if (f) {
        f->step_first = f->samples_done;
        f->step_samples = samples;
        f->step_rounds = samples > 0 ? rounds : 0;
        f->step_div = div;
        f->hyp_base = hyp_excl;
        P.sample_prefix[a] = s_excl;
    }
    if (a == 0) {
        P.sample_prefix[P.n_active] = total;
        P.counters[kCSamplesTotal] = (unsigned long long)total;
        P.counters[kCScoreNext] = 0;
        P.counters[kCRescoreNext] = 0;
        P.counters[kCCandNext] = 0;
        P.counters[kCStillRansac] = 0;
        P.counters[kCLMPending] = 0;
    }
}

// -------------------------------------------------------- sample + P3P -----
// One thread per minimal sample (replaces thread 0 of a 384-thread block in
// ransac.cuh:176-217). Solutions are appended to the frame's hypothesis region
// with one atomic per frame per warp; each carries id = sample*4 + solution,
// so ordering never depends on scheduling.
// One thread per sample draws its triple and finds its P3P candidates (the
// root filters); the warp then shares out the candidates -- 0 to 4 a sample --
// so that the depth polish and the pose, most of the arithmetic, run on full
// warps instead of once per candidate slot that any lane of the warp needs.
// Every candidate runs p3p_solve's own steps (p3p_finish) and keeps its order
// (hId = sample * 4 + solution); the compiler may fuse a multiply-add
// differently than in a per-thread loop, so poses can differ from that form in
// the last bits, never in which samples give solutions.
struct P3PStage {  // one lane's sample, staged for its warp
    P3PCtx c;
    double dep[12];
    int64_t h0, s;  // its first hypothesis slot, its sample id
    int a, n;       // active index of its frame, candidates
};
__global__ void __launch_bounds__(128) k_sample_p3p(Pools P) {
    __shared__ P3PStage stage[128];
    __shared__ int excl[128];
    const int64_t total = (int64_t)P.counters[kCSamplesTotal];
    const int lane = threadIdx.x & 31, wb = threadIdx.x & ~31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t g0 = (int64_t)blockIdx.x * blockDim.x; g0 < total; g0 += stride) {
        const int64_t g = g0 + threadIdx.x;
        const bool valid = g < total;
        P3PStage &me = stage[threadIdx.x];
        int a = -1;
        int nsol = 0;
        int64_t s = 0;
        if (valid) {
            a = find_segment(P.sample_prefix, P.n_active, g);
            const FrameDev &f = P.frames[P.active[a]];
            s = f.step_first + (g - P.sample_prefix[a]);
            int32_t idx[3];
            if (f.replay) {
                idx[0] = f.replay[3 * s];
                idx[1] = f.replay[3 * s + 1];
                idx[2] = f.replay[3 * s + 2];
            } else if (f.prosac) {
                prosac_triple(f.seed, (uint64_t)s, (uint32_t)f.n, P.prosac64 + f.blk_off * kSub, idx);
            } else {
                draw_triple(f.seed, (uint64_t)s, (uint32_t)f.n, idx);
            }
            const int64_t base = f.blk_off * kSub;
            d3 xb[3], Xs[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int64_t p = base + idx[k];
                xb[k] = bearing(P.xn64[2 * p], P.xn64[2 * p + 1]);
                Xs[k] = {P.X64[3 * p], P.X64[3 * p + 1], P.X64[3 * p + 2]};
            }
            nsol = p3p_candidates(xb, Xs, me.c, me.dep);
        }
        // Warp-aggregated reservation; a warp's samples are contiguous in g, so
        // lanes of one frame form one contiguous run.
        const unsigned act = __activemask();
        const unsigned grp = __match_any_sync(act, a);
        int incl = nsol;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(act, incl, o);
            if (lane >= o) incl += u;
        }
        const int first = __ffs(grp) - 1, last = 31 - __clz(grp);
        const int before = __shfl_sync(act, incl - nsol, first);
        const int grp_total = __shfl_sync(act, incl, last) - before;
        int slot0 = 0;
        if (lane == first && a >= 0 && grp_total > 0)
            slot0 = atomicAdd(&P.frames[P.active[a]].hyp_count, grp_total);
        slot0 = __shfl_sync(act, slot0, first);
        if (nsol > 0) me.h0 = P.frames[P.active[a]].hyp_base + slot0 + (incl - nsol - before);
        me.s = s;
        me.a = a;
        me.n = nsol;
        excl[threadIdx.x] = incl - nsol;
        const int T = __shfl_sync(0xffffffffu, incl, 31);  // the warp's candidates
        __syncwarp();
        for (int j = lane; j < T; j += 32) {
            // Owner: the last lane whose exclusive prefix is <= j.
            int lo = 0, hi = 31;
#pragma unroll
            for (int it = 0; it < 5; ++it) {
                const int mid = (lo + hi + 1) >> 1;
                if (excl[wb + mid] <= j) lo = mid; else hi = mid - 1;
            }
            const P3PStage &o = stage[wb + lo];
            const int k = j - excl[wb + lo];
            double S[12];
            p3p_finish(o.c, o.dep[3 * k], o.dep[3 * k + 1], o.dep[3 * k + 2], S);
            const FrameDev &f = P.frames[P.active[o.a]];
            const int64_t h = o.h0 + k;
            const double itau = 1.0 / f.tau;
#pragma unroll
            for (int e = 0; e < 12; ++e) P.hP64[12 * h + e] = S[e];
            P.hId[h] = o.s * 4 + k;
            // Scoring form: rows 0, 1 scaled by 1/tau, translation moved to the
            // centred frame (t + R c), all in FP64 before the FP32 rounding.
            float *Q = P.hP32 + 12 * h;
            float q32[12];
            bool finite = true;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const double tc = S[4 * r + 3] + S[4 * r] * f.centre[0] + S[4 * r + 1] * f.centre[1] +
                                  S[4 * r + 2] * f.centre[2];
                const double sc = r < 2 ? itau : 1.0;
                q32[4 * r] = (float)(S[4 * r] * sc);
                q32[4 * r + 1] = (float)(S[4 * r + 1] * sc);
                q32[4 * r + 2] = (float)(S[4 * r + 2] * sc);
                q32[4 * r + 3] = (float)(tc * sc);
            }
            // Rotation rows (scaled by 1/tau) within 2^40 and translations within
            // 2^80 keep every depth of a staged point (within 2^80) below 2^123:
            // no overflow, so no inf - inf and no NaN in the filter.
#pragma unroll
            for (int e = 0; e < 12; ++e)
                finite = finite && fabsf(q32[e]) <= ((e & 3) == 3 ? 0x1p80f : 0x1p40f);
            // A pose outside that range scores every point as an outlier
            // (depth -1, lateral offset 1).
#pragma unroll
            for (int e = 0; e < 12; ++e)
                Q[e] = finite ? q32[e] : (e == 3 || e == 7 ? 1.0f : (e == 11 ? -1.0f : 0.0f));
        }
        __syncwarp();  // the staging is reused by the next samples of this warp
    }
}

// ------------------------------------------------------------ scoring -----
// Work items: (frame, block of 32*HR hypotheses, point chunk). Chunks are sized
// so that the step has enough items to keep every SM busy.
__global__ void k_score_plan(Pools P) {
    __shared__ int64_t sh[33];
    __shared__ unsigned long long pairs_total;
    const int a = threadIdx.x;
    FrameDev *f = a < P.n_active ? &P.frames[P.active[a]] : nullptr;
    const bool act = f && f->step_samples > 0;
    if (a == 0) pairs_total = 0;
    __syncthreads();
    if (act) atomicAdd(&pairs_total, (unsigned long long)f->hyp_count * (unsigned long long)f->n);
    __syncthreads();
    __shared__ unsigned long long parts_total;
    if (a == 0) parts_total = 0;
    int64_t items = 0, parts = 0, hbs = 0;
    int HB = 32, nhb = 0, cb = 1;
    if (act) {
        HB = 32 * f->hr;
        nhb = (f->hyp_count + HB - 1) / HB;
        // About 8 items per warp slot of the GPU (FP32 kernels, one warp per
        // item) or per 4 CTA slots (the tensor-core kernel, a CTA per item with
        // a larger fixed cost per item); at least 2 staging blocks per item.
        const double target_items = f->hr == 1 ? 8.0 * P.num_sms * 4 : 8.0 * P.num_sms * 16;
        const double pairs_per_item = fmax((double)pairs_total / target_items, 2.0 * kSub * HB);
        cb = (int)ceil(pairs_per_item / ((double)HB * kSub));
        if (f->chunk_points > 0) cb = max(1, f->chunk_points / kSub);
        cb = max(cb, (f->n_blocks + kMaxScoreChunks - 1) / kMaxScoreChunks);
        cb = max(1, min(cb, f->n_blocks));
        atomicAdd(&parts_total, (unsigned long long)f->hyp_count * ((f->n_blocks + cb - 1) / cb));
    }
    __syncthreads();
    if (act) {
        // Keep the chunk partials within their buffer.
        const unsigned long long pt = parts_total;
        if (pt > (unsigned long long)P.max_parts) {
            const int scale = (int)((pt + P.max_parts - 1) / P.max_parts);
            cb = min(f->n_blocks, cb * scale);
        }
        const int nch = (f->n_blocks + cb - 1) / cb;
        f->n_hblocks = nhb;
        f->chunk_blocks = cb;
        f->n_chunks = nch;
        items = (int64_t)nhb * nch;
        parts = (int64_t)f->hyp_count * nch;
        hbs = nhb;
    }
    // Round minima of every planned frame, reset by the whole block.
    for (int idx = threadIdx.x; idx < P.n_active * kMaxRoundsPerStep; idx += blockDim.x) {
        FrameDev &g = P.frames[P.active[idx / kMaxRoundsPerStep]];
        if (g.step_samples > 0) g.round_min[idx % kMaxRoundsPerStep] = ~0ull;
    }
    int64_t tot;
    const int64_t iexcl = block_exclusive_scan(items, sh, tot);
    if (a < P.n_active) P.item_prefix[a] = iexcl;
    if (a == 0) {
        P.item_prefix[P.n_active] = tot;
        P.counters[kCScoreTotal] = (unsigned long long)tot;
        P.counters[kCWorkPairs] = pairs_total;
        P.counters[kCPairsTotal] += pairs_total;
    }
    const int64_t pexcl = block_exclusive_scan(parts, sh, tot);
    if (act) f->part_base = pexcl;
    if (a == 0 && tot > P.max_parts) flag_error(P, kErrOverflow);
    const int64_t hexcl = block_exclusive_scan(hbs, sh, tot);
    if (act) f->hb_base = hexcl;
    // The step's hypothesis-block arrival counters are [0, tot): zeroed by the block.
    for (int64_t i = threadIdx.x; i < min(tot, P.max_hb); i += blockDim.x) P.hb_arrive[i] = 0;
    if (a == 0 && tot > P.max_hb) flag_error(P, kErrOverflow);
}

// Per (hypothesis, point) the FP32 filter accumulates min(r^2 / tau^2, 1),
// counting a point with non-positive depth as an outlier (msac.cuh:46
// semantics) without a division or a branch: a depth below 2^-100 is raised
// to 2^-100 before the reciprocal, so the residual of a point behind the
// camera is ~2^100 x its lateral offset and saturates; the last FMA of r^2
// saturates to [0, 1] itself. Inputs are finite by construction (non-finite
// points and hypotheses are replaced when staged), so the saturating FMA never
// sees NaN. HP hypothesis pairs x PP points as independent packed-FP32 chains,
// staged so that every depth and its reciprocal issue first and the MUFU
// latency is covered by the other two rows: z2 -> rcp, then z0, z1, residuals,
// saturating r^2, sum.
template <int HP, int PP>
__device__ __forceinline__ void msac_chains(const uint64_t (&c)[HP][12], const uint64_t (&X)[PP],
                                            const uint64_t (&Y)[PP], const uint64_t (&Z)[PP],
                                            const uint64_t (&NX)[PP], const uint64_t (&NY)[PP], uint64_t (&acc)[HP]) {
    float ia[HP][PP], ib[HP][PP];
#pragma unroll
    for (int h = 0; h < HP; ++h)
#pragma unroll
        for (int p = 0; p < PP; ++p) {
            const uint64_t z2 = f2fma(c[h][8], X[p], f2fma(c[h][9], Y[p], f2fma(c[h][10], Z[p], c[h][11])));
            float za, zb;
            f2unpack(z2, za, zb);
            ia[h][p] = rcp_approx(fmaxf(za, kDepthFloor));
            ib[h][p] = rcp_approx(fmaxf(zb, kDepthFloor));
        }
#pragma unroll
    for (int h = 0; h < HP; ++h)
#pragma unroll
        for (int p = 0; p < PP; ++p) {
            const uint64_t z0 = f2fma(c[h][0], X[p], f2fma(c[h][1], Y[p], f2fma(c[h][2], Z[p], c[h][3])));
            const uint64_t z1 = f2fma(c[h][4], X[p], f2fma(c[h][5], Y[p], f2fma(c[h][6], Z[p], c[h][7])));
            const uint64_t inv = f2pack(ia[h][p], ib[h][p]);
            const uint64_t r0 = f2fma(z0, inv, NX[p]);
            const uint64_t r1 = f2fma(z1, inv, NY[p]);
            const uint64_t r1s = f2mul(r1, r1);
            float r0a, r0b, sa, sb;
            f2unpack(r0, r0a, r0b);
            f2unpack(r1s, sa, sb);
            acc[h] = f2add(acc[h], f2pack(fma_sat(r0a, r0a, sa), fma_sat(r0b, r0b, sb)));
        }
}

// One staging block (kSub points) against the lane's HP hypothesis pairs,
// PP points at a time (each 16-byte shared load carries two duplicated points).
template <int HP, int PP>
__device__ __forceinline__ void score_block(const float2 *blk, int valid, const uint64_t (&c)[HP][12],
                                            uint64_t (&acc)[HP]) {
    const ulonglong2 *sX = reinterpret_cast<const ulonglong2 *>(blk);
    const ulonglong2 *sY = sX + kSub / 2;
    const ulonglong2 *sZ = sY + kSub / 2;
    const ulonglong2 *sNX = sZ + kSub / 2;
    const ulonglong2 *sNY = sNX + kSub / 2;
    if (valid == kSub) {
#pragma unroll 1
        for (int j = 0; j < kSub / 2; j += PP / 2) {
            uint64_t X[PP], Y[PP], Z[PP], NX[PP], NY[PP];
#pragma unroll
            for (int k = 0; k < PP / 2; ++k) {
                const ulonglong2 x = sX[j + k], y = sY[j + k], z = sZ[j + k], nx = sNX[j + k], ny = sNY[j + k];
                X[2 * k] = x.x; X[2 * k + 1] = x.y;
                Y[2 * k] = y.x; Y[2 * k + 1] = y.y;
                Z[2 * k] = z.x; Z[2 * k + 1] = z.y;
                NX[2 * k] = nx.x; NX[2 * k + 1] = nx.y;
                NY[2 * k] = ny.x; NY[2 * k + 1] = ny.y;
            }
            msac_chains<HP, PP>(c, X, Y, Z, NX, NY, acc);
        }
    } else {
        const uint64_t *u = reinterpret_cast<const uint64_t *>(blk);
        for (int j = 0; j < valid; ++j) {
            uint64_t X[1] = {u[j]}, Y[1] = {u[kSub + j]}, Z[1] = {u[2 * kSub + j]}, NX[1] = {u[3 * kSub + j]},
                     NY[1] = {u[4 * kSub + j]};
            msac_chains<HP, 1>(c, X, Y, Z, NX, NY, acc);
        }
    }
}

// The FP32 filter pass. Persistent: each warp repeatedly takes a work item,
// streams its point chunk through a private two-stage shared-memory pipeline
// fed by 1-D bulk copies (TMA engine, mbarrier completion), and accumulates
// per-hypothesis truncated-MSAC costs for 32*HR hypotheses held in registers
// as packed FP32x2 pairs. The warp that completes the last chunk of a
// hypothesis block sums the chunk partials in fixed order and publishes the
// per-round minimum as a packed (score, index) key.
template <int HP, int PP>
__global__ void __launch_bounds__(kScoreWarps * 32) k_score(Pools P) {
    __shared__ __align__(128) float2 stage[kScoreWarps][2][kBlockFloat2];
    __shared__ __align__(8) uint64_t bars[kScoreWarps][2];
    constexpr int HR = 2 * HP;
    constexpr int HB = 32 * HR;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t *bar = bars[w];
    float2 *st0 = stage[w][0], *st1 = stage[w][1];
    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncwarp();
    uint32_t phase0 = 0, phase1 = 0;
    const int64_t total = (int64_t)P.counters[kCScoreTotal];
    const int64_t warps_total = (int64_t)gridDim.x * kScoreWarps;
    // Guided self-scheduling: a warp takes a run of consecutive items (chunks of
    // one hypothesis block in order), long while much work remains and single
    // items at the tail; hypotheses stay in registers while the run stays in
    // one block.
    int64_t run_next = 0, run_end = 0;
    int cur_a = -1, cur_hb = -1;
    uint64_t c[HP][12];
    for (;;) {
        if (run_next >= run_end) {
            int64_t start = 0, len = 0;
            if (lane == 0) {
                const int64_t done = (int64_t)*(volatile unsigned long long *)&P.counters[kCScoreNext];
                len = max((int64_t)1, min((int64_t)8, (total - done) / (4 * warps_total)));
                start = (int64_t)atomicAdd(&P.counters[kCScoreNext], (unsigned long long)len);
            }
            start = __shfl_sync(0xffffffffu, start, 0);
            len = __shfl_sync(0xffffffffu, len, 0);
            if (start >= total) break;
            run_next = start;
            run_end = min(total, start + len);
        }
        const int64_t item = run_next++;
        const int a = find_segment(P.item_prefix, P.n_active, item);
        FrameDev &f = P.frames[P.active[a]];
        const int64_t local = item - P.item_prefix[a];
        const int nch = f.n_chunks;
        const int hb = (int)(local / nch), ch = (int)(local % nch);
        const int nh = f.hyp_count;
        const int64_t hbase = f.hyp_base;
        // Hypotheses: lane owns HR consecutive ones (reloaded when the block changes).
        if (a != cur_a || hb != cur_hb) {
#pragma unroll
            for (int h = 0; h < HP; ++h) {
                const int i0 = hb * HB + lane * HR + 2 * h, i1 = i0 + 1;
                const float *A = P.hP32 + 12 * (hbase + i0), *Bp = P.hP32 + 12 * (hbase + i1);
#pragma unroll
                for (int e = 0; e < 12; ++e)
                    c[h][e] = f2pack(i0 < nh ? __ldg(A + e) : 0.0f, i1 < nh ? __ldg(Bp + e) : 0.0f);
            }
            cur_a = a;
            cur_hb = hb;
        }
        uint64_t acc[HP];
#pragma unroll
        for (int h = 0; h < HP; ++h) acc[h] = 0ull;
        const int b0 = ch * f.chunk_blocks;
        const int b1 = min(f.n_blocks, b0 + f.chunk_blocks);
        const int nb = b1 - b0;
        const float2 *g = P.pts32 + (f.blk_off + b0) * kBlockFloat2;
        if (lane == 0) {
            fence_proxy_async();
            bulk_load(st0, g, kBlockBytes, &bar[0]);
            if (nb > 1) bulk_load(st1, g + kBlockFloat2, kBlockBytes, &bar[1]);
        }
        bool ok = true;
        for (int i = 0; i < nb; ++i) {
            const int s = i & 1;
            const uint32_t ph = s ? phase1 : phase0;
            if (!mbar_wait(&bar[s], ph, kMaxPolls)) {
                ok = false;
                break;
            }
            if (s) phase1 ^= 1u; else phase0 ^= 1u;
            const int64_t pt0 = (int64_t)(b0 + i) * kSub;
            const int valid = (int)(f.n - pt0 < kSub ? f.n - pt0 : kSub);
            score_block<HP, PP>(s ? st1 : st0, valid, c, acc);
            __syncwarp();
            if (lane == 0 && i + 2 < nb) {
                fence_proxy_async();
                bulk_load(s ? st1 : st0, g + (int64_t)(i + 2) * kBlockFloat2, kBlockBytes, &bar[s]);
            }
        }
        if (!ok) {
            // Give up: record it, let any copy still in flight land, and leave.
            if (lane == 0) flag_error(P, kErrTimeout);
            mbar_wait(&bar[0], phase0, kMaxPolls);
            mbar_wait(&bar[1], phase1, kMaxPolls);
            return;
        }
        // Chunk partials.
        float *part = P.part + f.part_base;
#pragma unroll
        for (int h = 0; h < HP; ++h) {
            float lo, hi;
            f2unpack(acc[h], lo, hi);
            const int i0 = hb * HB + lane * HR + 2 * h;
            if (i0 < nh) part[(int64_t)i0 * nch + ch] = lo;
            if (i0 + 1 < nh) part[(int64_t)(i0 + 1) * nch + ch] = hi;
        }
        __threadfence();
        __syncwarp();
        unsigned prev = 0;
        if (lane == 0) prev = atomicAdd(&P.hb_arrive[f.hb_base + hb], 1u);
        prev = __shfl_sync(0xffffffffu, prev, 0);
        if (prev == (unsigned)(nch - 1)) {
            __threadfence();
            for (int k = 0; k < HR; ++k) {
                const int i = hb * HB + lane * HR + k;
                if (i >= nh) break;
                float s = 0.0f;
                for (int q = 0; q < nch; ++q) s += __ldcg(part + (int64_t)i * nch + q);
                P.hS32[hbase + i] = s;
                const int64_t sample = P.hId[hbase + i] >> 2;
                const int64_t r = (sample - f.step_first) / f.step_div;
                const unsigned long long key =
                    ((unsigned long long)__float_as_uint(s) << 32) | (unsigned)i;
                atomicMin(&f.round_min[r], key);
            }
        }
    }
}

// ------------------------------------------------ tensor-core scoring --
// The same filter with the projection on the 5th-generation tensor cores:
// for a tile of 128 points and a block of 32 hypotheses, one tcgen05.mma pair
// (kind::tf32, M = 128 points, N = 96 = z2 | z0 | z1 rows of the 32
// hypotheses, K = 16 in two steps of 8) writes every z of the tile into tensor
// memory, and the epilogue (one thread per point) does the reciprocal, the
// residuals, the saturating r^2 and the sum per hypothesis. TF32 keeps 11 significant bits,
// so each operand is split into a hi part (rounded to nearest TF32) and the
// rounded remainder, and the two MMA steps carry all four cross terms: both
// read the same A row (K = 8), the first with the hi, the second with the lo
// half of the hypothesis row
//   A row (point)      = [Xh Yh Zh 1 | Xl Yl Zl 0]
//   B row (hyp. row c) = [ch0..ch3   | ch0..ch2 0 | cl0..cl3   | cl0..cl2 0]
// whose products are exact in FP32 and sum to c . [X 1] with an error of the
// order of FP32 rounding (the remainders' own rounding is 2^-23 relative).
// The default scoring shape (FrameDev::hr = 1, points_per_iter = 128).
constexpr int kTcHyp = 32;        // hypotheses per item (HB at HR = 1)
constexpr int kTcN = 3 * kTcHyp;   // MMA N: z2 | z0 | z1 rows of the block
constexpr int kTcPts = 128;       // MMA M: points per tile
constexpr int kTcThreads = 128;   // one thread per point row of the accumulator
constexpr int kTcCols = 128;      // tensor-memory columns per CTA (four CTAs per SM at most)
constexpr int kTcPP = 128;        // points_per_iter value of the shape
// At most four CTAs per SM (so that 4 x 128 columns never exceed the 512 of an
// SM and tcgen05.alloc never waits): each asks for more than a fifth of the
// SM's shared memory. Four CTAs give the epilogue 16 warps per SM.
constexpr int kTcSmem = 48 * 1024;
constexpr uint32_t kTcIdesc = (1u << 4)                        // D: F32
                              | (2u << 7) | (2u << 10)         // A, B: TF32, both K-major
                              | ((uint32_t)(kTcN >> 3) << 17)  // N
                              | ((uint32_t)(kTcPts >> 4) << 24);  // M
// Shared-memory carve-up (bytes): A, B, two point-staging buffers (two
// blocks each), the cross-warp sums, then barriers and control words.
constexpr int kTcOffA = 0, kTcOffB = 8192, kTcOffPts = 14336, kTcOffRed = 24576, kTcOffCtl = 25088;

// Byte offset of element (row r, k) of a K-major operand with 16 K values per
// row, no swizzle: 8-row x 16-byte core matrices, the four K chunks of a row
// group adjacent (leading byte offset 128), row groups 512 bytes apart.
__device__ __forceinline__ int tc_off(int r, int k) {
    return (((r >> 3) * 4 + (k >> 2)) * 128) + (r & 7) * 16 + (k & 3) * 4;
}
// K-major operand with 8 K values per row (two 16-byte K chunks, leading byte
// offset 128, row groups 256 bytes apart).
__device__ __forceinline__ int tc_off8(int r, int k) {
    return (((r >> 3) * 2 + (k >> 2)) * 128) + (r & 7) * 16 + (k & 3) * 4;
}
__device__ __forceinline__ uint64_t tc_desc_sbo(const void *smem, uint32_t sbo) {
    return (uint64_t)((smem_addr(smem) >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
           ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}
__device__ __forceinline__ uint64_t tc_desc(const void *smem) {
    return (uint64_t)((smem_addr(smem) >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
           ((uint64_t)(512 >> 4) << 32) | (1ull << 46);
}
__device__ __forceinline__ float tf32_rn(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    const uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kTcIdesc), "r"(accumulate), "r"(m0), "r"(m1), "r"(m2), "r"(m3));
}
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// B operand of hypothesis block hb: thread t < 32 writes the z2, z0 and z1 rows
// (t, 32 + t, 64 + t) of hypothesis hb * 32 + t (zero rows past the count).
__device__ __forceinline__ void tc_build_b(float *sB, const Pools &P, const FrameDev &f, int hb) {
    const int t = threadIdx.x;
    if (t >= kTcHyp) return;
    const int i = hb * kTcHyp + t;
    const float *src = P.hP32 + 12 * (f.hyp_base + i);
    float c[12];
#pragma unroll
    for (int e = 0; e < 12; ++e) c[e] = i < f.hyp_count ? __ldg(src + e) : 0.0f;
    char *rb = reinterpret_cast<char *>(sB);
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
        const int n = comp * kTcHyp + t;
        const int cb = comp == 0 ? 8 : (comp == 1 ? 0 : 4);  // z2 | z0 | z1
        float hi[4], lo[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            hi[k] = tf32_rn(c[cb + k]);
            lo[k] = tf32_rn(c[cb + k] - hi[k]);
        }
        *reinterpret_cast<float4 *>(rb + tc_off(n, 0)) = make_float4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<float4 *>(rb + tc_off(n, 4)) = make_float4(hi[0], hi[1], hi[2], 0.0f);
        *reinterpret_cast<float4 *>(rb + tc_off(n, 8)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
        *reinterpret_cast<float4 *>(rb + tc_off(n, 12)) = make_float4(lo[0], lo[1], lo[2], 0.0f);
    }
}

__global__ void __launch_bounds__(kTcThreads, 4) k_score_tc(Pools P) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    float *sA = reinterpret_cast<float *>(tc_smem + kTcOffA);
    float *sB = reinterpret_cast<float *>(tc_smem + kTcOffB);
    float2 *sPts = reinterpret_cast<float2 *>(tc_smem + kTcOffPts);  // 2 buffers x 2 staging blocks
    float *red = reinterpret_cast<float *>(tc_smem + kTcOffRed);      // [4][32]
    uint64_t *bars = reinterpret_cast<uint64_t *>(tc_smem + kTcOffCtl);  // points 0, 1; MMA
    uint32_t *tslot = reinterpret_cast<uint32_t *>(tc_smem + kTcOffCtl + 32);
    int *ctl = reinterpret_cast<int *>(tc_smem + kTcOffCtl + 48);
    volatile int *err = reinterpret_cast<volatile int *>(tc_smem + kTcOffCtl + 60);  // a wait gave up
    long long *run = reinterpret_cast<long long *>(tc_smem + kTcOffCtl + 64);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) {
        *err = 0;
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        fence_mbar_init();
    }
    if (w == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                     "r"((uint32_t)kTcCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t trow = tmem + ((uint32_t)(w * 32) << 16);  // this warp's 32 lanes
    uint32_t ph0 = 0, ph1 = 0, phm = 0;
    const int64_t total = (int64_t)P.counters[kCScoreTotal];
    const int64_t ctas = gridDim.x;
    int cur_a = -1, cur_hb = -1;
    int64_t run_next = 0, run_end = 0;
    bool ok = true;
    for (;;) {
        if (run_next >= run_end) {
            if (tid == 0) {
                const int64_t done = (int64_t)*(volatile unsigned long long *)&P.counters[kCScoreNext];
                const int64_t len = max((int64_t)1, min((int64_t)8, (total - done) / (4 * ctas)));
                run[0] = (long long)atomicAdd(&P.counters[kCScoreNext], (unsigned long long)len);
                run[1] = len;
            }
            __syncthreads();
            const int64_t start = run[0], len = run[1];
            __syncthreads();
            if (start >= total) break;
            run_next = start;
            run_end = min(total, start + len);
        }
        const int64_t item = run_next++;
        const int a = find_segment(P.item_prefix, P.n_active, item);
        FrameDev &f = P.frames[P.active[a]];
        const int64_t local = item - P.item_prefix[a];
        const int nch = f.n_chunks;
        const int hb = (int)(local / nch), ch = (int)(local % nch);
        const int nh = f.hyp_count;
        if (a != cur_a || hb != cur_hb) {  // every MMA of the previous item has completed
            tc_build_b(sB, P, f, hb);
            cur_a = a;
            cur_hb = hb;
        }
        const int b0 = ch * f.chunk_blocks;
        const int b1 = min(f.n_blocks, b0 + f.chunk_blocks);
        const int ntiles = (b1 - b0 + 1) / 2;
        const int64_t fn = f.n;  // read once: the asm barriers below would reload it every tile
        const float2 *g = P.pts32 + (f.blk_off + b0) * kBlockFloat2;
        auto tile_blocks = [&](int i) { return min(2, b1 - b0 - 2 * i); };
        if (tid == 0) {
            fence_proxy_async();
            bulk_load(sPts, g, (uint32_t)(tile_blocks(0) * kBlockBytes), &bars[0]);
            if (ntiles > 1)
                bulk_load(sPts + 2 * kBlockFloat2, g + 2 * kBlockFloat2, (uint32_t)(tile_blocks(1) * kBlockBytes),
                          &bars[1]);
        }
        uint64_t acc[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[j] = 0ull;
        // Every thread waits on the copy and MMA barriers itself (two CTA
        // barriers per tile). A wait that gives up records the error and the
        // thread carries on through the same barriers, so the CTA leaves the
        // tile loop together once the error is visible to all.
        for (int i = 0; i < ntiles; ++i) {
            const int s = i & 1;
            if (!*err && !mbar_wait(&bars[s], s ? ph1 : ph0, kMaxPolls)) *err = 1;
            if (s) ph1 ^= 1u; else ph0 ^= 1u;
            // A row of this thread's point.
            const int64_t p0 = (int64_t)(b0 + 2 * i) * kSub;
            const int cnt = (int)min((int64_t)tile_blocks(i) * kSub, fn - p0);
            const bool v = tid < cnt;
            const float2 *tb = sPts + s * 2 * kBlockFloat2 + (tid >> 6) * kBlockFloat2;
            const int j = tid & (kSub - 1);
            const float X = v ? tb[j].x : 0.0f, Y = v ? tb[kSub + j].x : 0.0f, Z = v ? tb[2 * kSub + j].x : 0.0f;
            const float NX = v ? tb[3 * kSub + j].x : 0.0f, NY = v ? tb[4 * kSub + j].x : 0.0f;
            {
                const float xh = tf32_rn(X), yh = tf32_rn(Y), zh = tf32_rn(Z);
                const float xl = tf32_rn(X - xh), yl = tf32_rn(Y - yh), zl = tf32_rn(Z - zh);
                const float one = v ? 1.0f : 0.0f;
                // K = 8 (the two MMAs read the same A chunks with the hi and the
                // lo half of the hypothesis rows): row groups 256 bytes apart.
                char *ra = reinterpret_cast<char *>(sA);
                *reinterpret_cast<float4 *>(ra + tc_off8(tid, 0)) = make_float4(xh, yh, zh, one);
                *reinterpret_cast<float4 *>(ra + tc_off8(tid, 4)) = make_float4(xl, yl, zl, 0.0f);
            }
            fence_proxy_async();  // the operands, written by threads, are read by the tensor core
            __syncthreads();      // the A tile is complete; staging buffer s is free
            if (tid == 0) {
                tc_fence_after();
                const uint64_t da = tc_desc_sbo(sA, 256);
                tc_mma(tmem, da, tc_desc(sB), 0u);
                tc_mma(tmem, da, tc_desc(reinterpret_cast<char *>(sB) + 256), 1u);
                tc_commit(&bars[2]);
                if (i + 2 < ntiles) {
                    fence_proxy_async();
                    bulk_load(sPts + s * 2 * kBlockFloat2, g + (int64_t)(2 * (i + 2)) * kBlockFloat2,
                              (uint32_t)(tile_blocks(i + 2) * kBlockBytes), &bars[s]);
                }
            }
            if (!*err && !mbar_wait(&bars[2], phm, kMaxPolls)) *err = 1;
            phm ^= 1u;
            tc_fence_after();
            const uint64_t nx2 = f2pack(NX, NX), ny2 = f2pack(NY, NY);
#pragma unroll
            for (int gq = 0; gq < 2; ++gq) {
                float z2[16], z0[16], z1[16];
                tc_ld16(trow + (uint32_t)(16 * gq), z2);
                tc_ld16(trow + (uint32_t)(kTcHyp + 16 * gq), z0);
                tc_ld16(trow + (uint32_t)(2 * kTcHyp + 16 * gq), z1);
                tc_wait_ld();
                if (v) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const float ia = rcp_approx(fmaxf(z2[2 * q], kDepthFloor));
                        const float ib = rcp_approx(fmaxf(z2[2 * q + 1], kDepthFloor));
                        const uint64_t inv = f2pack(ia, ib);
                        const uint64_t r0 = f2fma(f2pack(z0[2 * q], z0[2 * q + 1]), inv, nx2);
                        const uint64_t r1 = f2fma(f2pack(z1[2 * q], z1[2 * q + 1]), inv, ny2);
                        const uint64_t r1s = f2mul(r1, r1);
                        float r0a, r0b, sa, sb;
                        f2unpack(r0, r0a, r0b);
                        f2unpack(r1s, sa, sb);
                        acc[8 * gq + q] = f2add(acc[8 * gq + q], f2pack(fma_sat(r0a, r0a, sa), fma_sat(r0b, r0b, sb)));
                    }
                }
            }
            tc_fence_before();
            __syncthreads();  // the accumulator and the A tile are free for the next tile
        }
        if (*err) ok = false;  // written before the last barrier, so every thread reads the same
        if (!ok) break;
        // Chunk partials: the warp's 32 hypotheses over its 32 points (lanes
        // 2p, 2p + 1 end with hypotheses 2p, 2p + 1), then the four warps in
        // fixed order.
#pragma unroll
        for (int o = 16, m = 8; o >= 2; o >>= 1, m >>= 1) {
            const bool up = (lane & o) != 0;
#pragma unroll
            for (int jj = 0; jj < m; ++jj) {
                const uint64_t keep = up ? acc[m + jj] : acc[jj];
                const uint64_t send = up ? acc[jj] : acc[m + jj];
                acc[jj] = f2add(keep, __shfl_xor_sync(0xffffffffu, send, o));
            }
        }
        acc[0] = f2add(acc[0], __shfl_xor_sync(0xffffffffu, acc[0], 1));
        if ((lane & 1) == 0) {
            float lo, hi;
            f2unpack(acc[0], lo, hi);
            red[w * kTcHyp + lane] = lo;
            red[w * kTcHyp + lane + 1] = hi;
        }
        __syncthreads();
        float *part = P.part + f.part_base;
        if (tid < kTcHyp) {
            const int i = hb * kTcHyp + tid;
            const float s4 = ((red[tid] + red[kTcHyp + tid]) + red[2 * kTcHyp + tid]) + red[3 * kTcHyp + tid];
            if (i < nh) part[(int64_t)i * nch + ch] = s4;
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) ctl[2] = (int)atomicAdd(&P.hb_arrive[f.hb_base + hb], 1u);
        __syncthreads();
        if (ctl[2] == nch - 1 && tid < kTcHyp) {
            __threadfence();
            const int i = hb * kTcHyp + tid;
            if (i < nh) {
                float s = 0.0f;
                for (int q = 0; q < nch; ++q) s += __ldcg(part + (int64_t)i * nch + q);
                P.hS32[f.hyp_base + i] = s;
                const int64_t sample = P.hId[f.hyp_base + i] >> 2;
                const int64_t r = (sample - f.step_first) / f.step_div;
                const unsigned long long key = ((unsigned long long)__float_as_uint(s) << 32) | (unsigned)i;
                atomicMin(&f.round_min[r], key);
            }
        }
        __syncthreads();  // red and ctl are reused by the next item
    }
    if (!ok) {
        // Give up: record it and let the copies and the MMA in flight land
        // (bounded) before the tensor memory is released.
        if (tid == 0) {
            flag_error(P, kErrTimeout);
            // Copies still in flight complete the buffers' current phases; the
            // last MMA issued completes the phase before the current parity.
            mbar_wait(&bars[0], ph0, kMaxPolls);
            mbar_wait(&bars[1], ph1, kMaxPolls);
            mbar_wait(&bars[2], phm ^ 1u, kMaxPolls);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (w == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTcCols));
}

// ---------------------------------------------------------- candidates -----
// Candidates for the exact FP64 re-rank: every hypothesis whose FP32 score s
// lies within a band of the running minimum thr of its round (over this
// step's rounds so far and the best of earlier steps), s <= thr + thr/4096 + 1
// (scores in tau^2 units). The FP32 score of a hypothesis is within 1e-5 of
// its FP64 score relative (tested), so the FP64 best of every round that can
// change the running best -- including every exact tie -- lies inside the
// safe band thr + thr/32768 + 1/2, twice that error on both sides with an
// absolute margin, and the candidate band contains the safe band. The band is
// never narrowed. When more than kMaxCandFrame hypotheses fall inside it:
//   * a step of several rounds (forced mode: more than kSplitSamples samples)
//     is redone: the frame's later steps are limited to the rounds that the
//     step's candidate rate leaves room for (half the cap, and fewer rounds
//     than the redone step, so repeated redos end at one round, which bounds
//     the candidates by 4 * B; forced: kSplitSamples samples), and k_finalize
//     discards this step; every step that fits then re-sizes the limit from
//     its own rate, up or down. A frame's samples, selection and stop
//     point do not depend on how its rounds are grouped into steps, so this
//     changes no result;
//   * a single round (B > kMaxCandFrame / 4) keeps the kMaxCandFrame smallest
//     keys (margin above thr in safe-band units, then sample id): the same
//     subset on every run, alone or in a mix; if that drops a hypothesis
//     inside the safe band, the frame's overflow flag is raised.
// A step whose candidates do not fit the step's shared pool is redone as
// well (the pool is claimed in launch order, which only delays a frame).
constexpr int kSplitSamples = kMaxCandFrame / 4;
__device__ __forceinline__ unsigned long long cand_key(float s, float t, float inv_safe, int64_t id,
                                                       int64_t first) {
    const float u = fmaxf((s - t) * inv_safe, 0.0f);
    return ((unsigned long long)__float_as_uint(u) << 32) | (unsigned long long)(uint32_t)(id - 4 * first);
}

__global__ void k_select(Pools P) {
    __shared__ float thr[kMaxRoundsPerStep], inv_safe[kMaxRoundsPerStep];
    __shared__ int rh[kMaxRoundsPerStep];
    __shared__ unsigned hist[256];
    __shared__ int cnt0, fill, mode, drop_safe;
    __shared__ unsigned need;
    __shared__ unsigned long long kstar;
    __shared__ long long base;
    const int slot = P.active[blockIdx.x];
    FrameDev &f = P.frames[slot];
    if (f.status != kRansac || f.step_samples == 0) return;
    const int R = (int)f.step_rounds;
    if (threadIdx.x == 0) {
        float pm = f.found ? (float)(f.best_score / f.sq_thr) : __int_as_float(0x7f800000);
        for (int r = 0; r < R; ++r) {
            const unsigned long long k = f.round_min[r];
            const float rm = k == ~0ull ? __int_as_float(0x7f800000) : __uint_as_float((unsigned)(k >> 32));
            pm = fminf(pm, rm);
            thr[r] = pm;
            inv_safe[r] = __frcp_rn(pm * (1.0f / 32768.0f) + 0.5f);
        }
        cnt0 = 0;
        fill = 0;
        drop_safe = 0;
    }
    for (int r = threadIdx.x; r < kMaxRoundsPerStep; r += blockDim.x) rh[r] = 0;
    __syncthreads();
    const int nh = f.hyp_count;
    const int64_t hb = f.hyp_base;
    int my = 0;
    for (int i = threadIdx.x; i < nh; i += blockDim.x) {
        const float s = P.hS32[hb + i];
        const int64_t r = ((P.hId[hb + i] >> 2) - f.step_first) / f.step_div;
        const float pm = thr[r];
        atomicAdd(&rh[r], 1);
        my += (s <= pm + (pm * (1.0f / 4096.0f) + 1.0f)) ? 1 : 0;
    }
    my = warp_sum(my);
    if ((threadIdx.x & 31) == 0) atomicAdd(&cnt0, my);
    __syncthreads();
    for (int r = threadIdx.x; r < kMaxRoundsPerStep; r += blockDim.x) f.round_hyps[r] = rh[r];
    if (threadIdx.x == 0) {
        const bool forced = f.force_samples > 0;
        const bool splittable = forced ? f.step_samples > kSplitSamples : f.step_rounds > 1;
        int want = cnt0, md = 0;                 // 0: every candidate
        if (cnt0 > kMaxCandFrame) {
            if (splittable) {
                // Later steps run at most as many rounds as this step's
                // candidate rate leaves room for with a margin of two, and
                // fewer than this step's, so that repeated redos end at one
                // round (forced mode: kSplitSamples samples).
                f.split = forced ? kSplitSamples
                                 : (int)max(1LL, min((long long)R - 1, (long long)kMaxCandFrame * R / (2LL * cnt0)));
                want = 0;
                md = 2;                          // redo the step
            } else {
                want = kMaxCandFrame;
                md = 1;                          // the smallest keys
            }
        }
        long long b0 = 0;
        if (want > 0) {
            b0 = (long long)atomicAdd(&P.counters[kCCandNext], (unsigned long long)want);
            if (b0 + want > P.cand_cap) {        // the step's pool is exhausted: redo
                want = 0;
                md = 2;
            }
        }
        if (md == 2) {
            f.redo = 1;
        } else if (!forced && f.split > 0) {
            // A step that fit after a redo: its candidate rate sizes the next
            // ones (margin of two), up as well as down, since the rate falls
            // once a good model has been found.
            f.split = (int)min((long long)kMaxRoundsPerStep,
                               max(1LL, (long long)kMaxCandFrame * R / (2LL * max(cnt0, 1))));
        }
        mode = md;
        need = (unsigned)want;
        kstar = ~0ull;
        base = b0;
        f.cand_base = b0;
        f.cand_count = want;
    }
    __syncthreads();
    if (mode == 2 || need == 0) return;
    if (mode == 1) {
        // Radix select (8 bits per pass) of the need-th smallest key among
        // the candidates; keys are distinct (the id part), so exactly `need`
        // keys are <= kstar.
        unsigned long long prefix = 0;
        for (int pass = 0; pass < 8; ++pass) {
            const int shift = 56 - 8 * pass;
            const unsigned long long hi_mask = pass == 0 ? 0ull : (~0ull << (shift + 8));
            for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
            __syncthreads();
            for (int i = threadIdx.x; i < nh; i += blockDim.x) {
                const float s = P.hS32[hb + i];
                const int64_t id = P.hId[hb + i];
                const int64_t r = ((id >> 2) - f.step_first) / f.step_div;
                const float pm = thr[r];
                if (!(s <= pm + (pm * (1.0f / 4096.0f) + 1.0f))) continue;
                const unsigned long long key = cand_key(s, pm, inv_safe[r], id, f.step_first);
                if ((key & hi_mask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                unsigned cum = 0, want_rank = need;
                int b = 0;
                for (; b < 255; ++b) {
                    if (cum + hist[b] >= want_rank) break;
                    cum += hist[b];
                }
                need = want_rank - cum;
                kstar = prefix | ((unsigned long long)b << shift);
            }
            __syncthreads();
            prefix = kstar;
        }
    }
    const unsigned long long kmax = mode == 1 ? kstar : ~0ull;
    const int cap = f.cand_count;
    for (int i = threadIdx.x; i < nh; i += blockDim.x) {
        const float s = P.hS32[hb + i];
        const int64_t id = P.hId[hb + i];
        const int64_t r = ((id >> 2) - f.step_first) / f.step_div;
        const float pm = thr[r];
        if (!(s <= pm + (pm * (1.0f / 4096.0f) + 1.0f))) continue;
        if (mode == 1) {
            const unsigned long long key = cand_key(s, pm, inv_safe[r], id, f.step_first);
            if (key > kmax) {
                if (__uint_as_float((unsigned)(key >> 32)) <= 1.0f) drop_safe = 1;
                continue;
            }
        }
        const int c = atomicAdd(&fill, 1);
        if (c < cap) P.cHyp[base + c] = i;
    }
    __syncthreads();
    if (threadIdx.x == 0 && drop_safe) f.overflow = 1;
}

__global__ void k_rescore_plan(Pools P) {
    __shared__ int64_t sh[33];
    const int a = threadIdx.x;
    int64_t items = 0;
    if (a < P.n_active) {
        const int slot = P.active[a];
        FrameDev &f = P.frames[slot];
        if (f.status == kRansac && f.step_samples > 0) {
            const int64_t want = (f.n + 2047) / 2048;
            const int nrc = (int)(want < kMaxRChunks ? want : kMaxRChunks);
            f.n_rchunks = nrc;
            f.rchunk = (f.n + nrc - 1) / nrc;
            items = (int64_t)((f.cand_count + kRescoreGroup - 1) / kRescoreGroup) * nrc;
        }
    }
    // The step's candidates lie in [0, claimed) of the pool: arrival counters zeroed by the block.
    const int64_t claimed = min((int64_t)P.counters[kCCandNext], P.cand_cap);
    for (int64_t c = threadIdx.x; c < claimed; c += blockDim.x) P.c_arrive[c] = 0;
    int64_t tot;
    const int64_t ex = block_exclusive_scan(items, sh, tot);
    if (a < P.n_active) P.ritem_prefix[a] = ex;
    if (a == 0) {
        P.ritem_prefix[P.n_active] = tot;
        P.counters[kCRescoreTotal] = (unsigned long long)tot;
    }
}

// Exact FP64 truncated MSAC of a group of up to kRescoreGroup candidates of a
// frame over one point chunk (the chunk's points are read once for the group),
// with the per-point formula of msac.cuh:18-56 (reciprocal of the depth, then
// products). Every candidate's sum has the same fixed order whatever the
// grouping: per thread the strided points, then the warp tree, the warps in
// order, and the chunks in order by the last chunk to finish, which adds
// (n - count) * tau^2 (ransac.cuh:322).
__global__ void __launch_bounds__(256) k_rescore(Pools P) {
    constexpr int G = kRescoreGroup;
    __shared__ double ss[8][G];
    __shared__ int sc[8][G];
    __shared__ double sM[G][12];
    __shared__ int64_t s_item;
    __shared__ unsigned s_prev[G];
    const int64_t total = (int64_t)P.counters[kCRescoreTotal];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int64_t)atomicAdd(&P.counters[kCRescoreNext], 1ull);
        __syncthreads();
        const int64_t item = s_item;
        if (item >= total) break;
        const int a = find_segment(P.ritem_prefix, P.n_active, item);
        const int slot = P.active[a];
        const FrameDev &f = P.frames[slot];
        const int64_t local = item - P.ritem_prefix[a];
        const int gi = (int)(local / f.n_rchunks), ch = (int)(local % f.n_rchunks);
        const int c0 = gi * G, ng = min(G, f.cand_count - c0);
        if (threadIdx.x < G * 12) {
            const int g = threadIdx.x / 12, e = threadIdx.x % 12;
            sM[g][e] = g < ng ? P.hP64[12 * (f.hyp_base + P.cHyp[f.cand_base + c0 + g]) + e] : 0.0;
        }
        __syncthreads();
        const int64_t base = f.blk_off * kSub;
        const int64_t p0 = (int64_t)ch * f.rchunk, p1 = (f.n < p0 + f.rchunk ? f.n : p0 + f.rchunk);
        double s[G];
        int cnt[G];
#pragma unroll
        for (int g = 0; g < G; ++g) {
            s[g] = 0.0;
            cnt[g] = 0;
        }
        const double sq = f.sq_thr;
        for (int64_t i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
            const int64_t p = base + i;
            const double X0 = P.X64[3 * p], X1 = P.X64[3 * p + 1], X2 = P.X64[3 * p + 2];
            const double x0 = P.xn64[2 * p], x1 = P.xn64[2 * p + 1];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                if (g < ng) {
                    const double *M = sM[g];
                    const double z0 = M[0] * X0 + M[1] * X1 + M[2] * X2 + M[3];
                    const double z1 = M[4] * X0 + M[5] * X1 + M[6] * X2 + M[7];
                    const double z2 = M[8] * X0 + M[9] * X1 + M[10] * X2 + M[11];
                    const double inv_z2 = 1.0 / z2;
                    const double r0 = z0 * inv_z2 - x0;
                    const double r1 = z1 * inv_z2 - x1;
                    const double r_sq = r0 * r0 + r1 * r1;
                    if (r_sq < sq && z2 > 0.0) {
                        s[g] += r_sq;
                        ++cnt[g];
                    }
                }
            }
        }
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const double sw = warp_sum(s[g]);
            const int cw = warp_sum(cnt[g]);
            if (lane == 0) {
                ss[warp][g] = sw;
                sc[warp][g] = cw;
            }
        }
        __syncthreads();
        if (threadIdx.x < ng) {
            const int g = threadIdx.x;
            const int64_t cs = f.cand_base + c0 + g;
            double S = 0.0;
            int C = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
                S += ss[k][g];
                C += sc[k][g];
            }
            P.cpS[cs * kMaxRChunks + ch] = S;
            P.cpC[cs * kMaxRChunks + ch] = C;
            __threadfence();
            s_prev[g] = atomicAdd(&P.c_arrive[cs], 1u);
            if (s_prev[g] == (unsigned)(f.n_rchunks - 1)) {
                __threadfence();
                double St = 0.0;
                int64_t Ct = 0;
                for (int q = 0; q < f.n_rchunks; ++q) {
                    St += __ldcg(P.cpS + cs * kMaxRChunks + q);
                    Ct += __ldcg(P.cpC + cs * kMaxRChunks + q);
                }
                P.cS64[cs] = St + (double)(f.n - Ct) * sq;
                P.cCnt[cs] = Ct;
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ finalize -----
// The reference's per-round bookkeeping (turbo_ransac.cu:176-257 with the
// merge/argmin kernels ransac.cuh:41-137), replayed in round order on the
// exact FP64 scores: a round's best (lowest score, then lowest sample and
// solution) replaces the running best only if strictly better; after each
// round the stop rule uses the running best's inlier count. One CTA per frame:
// the per-round minima are found in parallel, the round walk is sequential.
__global__ void __launch_bounds__(256) k_finalize(Pools P) {
    __shared__ unsigned long long rmin[kMaxRoundsPerStep];   // ordered FP64 score
    __shared__ unsigned long long rid[kMaxRoundsPerStep];    // hypothesis id
    __shared__ int rwin[kMaxRoundsPerStep];                  // candidate index
    const int slot = P.active[blockIdx.x];
    FrameDev &f = P.frames[slot];
    if (f.status != kRansac) return;
    if (f.step_samples == 0) {  // waiting for hypothesis capacity
        if (threadIdx.x == 0) atomicAdd(&P.counters[kCStillRansac], 1ull);
        return;
    }
    const int redo = f.redo;
    __syncthreads();
    if (redo) {  // the step's re-rank candidates did not fit (k_select): its rounds run again
        if (threadIdx.x == 0) {
            f.redo = 0;
            f.steps += 1;
            atomicAdd(&P.counters[kCStillRansac], 1ull);
        }
        return;
    }
    for (int r = threadIdx.x; r < kMaxRoundsPerStep; r += blockDim.x) {
        rmin[r] = ~0ull;
        rid[r] = ~0ull;
        rwin[r] = -1;
    }
    __syncthreads();
    const int C = f.cand_count;
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        const int64_t id = P.hId[f.hyp_base + P.cHyp[f.cand_base + c]];
        const int64_t r = ((id >> 2) - f.step_first) / f.step_div;
        atomicMin(&rmin[r], dbl_to_ordered(P.cS64[f.cand_base + c]));
    }
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        const int64_t id = P.hId[f.hyp_base + P.cHyp[f.cand_base + c]];
        const int64_t r = ((id >> 2) - f.step_first) / f.step_div;
        if (dbl_to_ordered(P.cS64[f.cand_base + c]) == rmin[r]) atomicMin(&rid[r], (unsigned long long)id);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        const int64_t id = P.hId[f.hyp_base + P.cHyp[f.cand_base + c]];
        const int64_t r = ((id >> 2) - f.step_first) / f.step_div;
        if ((unsigned long long)id == rid[r]) rwin[r] = c;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    f.rescored += C;
    const bool forced = f.force_samples > 0;
    bool stop = false;
    int64_t r_end = f.step_rounds;
    for (int64_t r = 0; r < f.step_rounds; ++r) {
        const int c = rwin[r];
        if (c >= 0) {
            const int64_t cs = f.cand_base + c;
            const double bs = P.cS64[cs];
            if (!f.found || bs < f.best_score) {
                const int64_t bid = (int64_t)rid[r];
                f.found = 1;
                f.best_score = bs;
                f.best_count = P.cCnt[cs];
                f.best_sample = bid >> 2;
                f.best_sol = (int32_t)(bid & 3);
                const double *Pp = P.hP64 + 12 * (f.hyp_base + P.cHyp[cs]);
                for (int e = 0; e < 12; ++e) f.best_P[e] = Pp[e];
            }
        }
        if (forced) continue;
        const int64_t after = f.step_first + (r + 1) * f.B;
        const int64_t need = needed_samples(f.found ? f.best_count : 0, f.n, f.log_missing, f.trials_mult, f.quirk);
        if ((after > need && after >= f.min_samples) || after >= f.max_total) {
            stop = true;
            r_end = r + 1;
            break;
        }
    }
    // Hypotheses of the rounds actually consumed.
    int64_t hyps = 0;
    for (int64_t r = 0; r < r_end; ++r) hyps += f.round_hyps[r];
    f.hyps_done += hyps;
    f.steps += 1;
    if (forced) {
        f.samples_done += f.step_samples;
        f.rounds_done += 1;
        if (f.samples_done >= f.force_samples) stop = true;
    } else {
        f.samples_done = f.step_first + r_end * f.B;
        f.rounds_done += r_end;
    }
    if (stop) {
        // Publish the best pose and the epoch before the status: k_inliers may
        // run concurrently on another stream and reads them in reverse order.
        f.lm_epoch = (int64_t)P.counters[kCSteps];
        __threadfence();
        *(volatile int32_t *)&f.status = kLMReady;
        atomicAdd(&P.counters[kCLMPending], 1ull);
    } else {
        atomicAdd(&P.counters[kCStillRansac], 1ull);
    }
}

// ------------------------------------------------------------- inliers -----
// get_inliers_mx (entry.cu:12-26) with the pose entry.cu:79-83 builds from the
// RANSAC result (R -> quaternion -> R), then an ordered compaction of the
// inliers into the LM arrays in pixel/f units (entry.cu:87-103).
__global__ void __launch_bounds__(1024) k_inliers(Pools P) {
    __shared__ int64_t sh[33];
    __shared__ double sR[9], st[3], sq[4];
    const int slot = P.active[blockIdx.x];
    FrameDev &f = P.frames[slot];
    __shared__ int take;
    if (threadIdx.x == 0) {
        const int32_t st0 = *(volatile int32_t *)&f.status;
        __threadfence();
        const int64_t ep = *(volatile int64_t *)&f.lm_epoch;
        take = (st0 == kLMReady && ep < (int64_t)*(volatile unsigned long long *)&P.counters[kCSteps]) ? 1 : 0;
        __threadfence();
    }
    __syncthreads();
    if (!take) return;
    if (threadIdx.x == 0) {
        double R[9];
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c) R[3 * r + c] = f.found ? f.best_P[4 * r + c] : (r == c ? 1.0 : 0.0);
            st[r] = f.found ? f.best_P[4 * r + 3] : 0.0;
        }
        double q[4];
        rotmat_to_quat(R, q);
        quat_to_rotmat(q, sR);
        for (int k = 0; k < 4; ++k) sq[k] = q[k];
    }
    __syncthreads();
    const int64_t base = f.blk_off * kSub;
    const double sqthr = f.sq_thr;
    const double scale = 1.0 / f.focal;  // entry.cu:87,98
    int64_t written = 0;
    for (int64_t i0 = 0; i0 < f.n; i0 += blockDim.x) {
        const int64_t i = i0 + threadIdx.x;
        int in = 0;
        if (i < f.n) {
            const int64_t p = base + i;
            const double X0 = P.X64[3 * p], X1 = P.X64[3 * p + 1], X2 = P.X64[3 * p + 2];
            const double Z0 = sR[0] * X0 + sR[1] * X1 + sR[2] * X2 + st[0];
            const double Z1 = sR[3] * X0 + sR[4] * X1 + sR[5] * X2 + st[1];
            const double Z2 = sR[6] * X0 + sR[7] * X1 + sR[8] * X2 + st[2];
            const double h0 = Z0 / Z2 - P.xn64[2 * p], h1 = Z1 / Z2 - P.xn64[2 * p + 1];
            const double r2 = h0 * h0 + h1 * h1;
            in = (r2 < sqthr && Z2 > 0.0) ? 1 : 0;
            P.mask[p] = (uint8_t)in;
        }
        int64_t tot;
        const int64_t ex = block_exclusive_scan(in, sh, tot);
        if (in) {
            const int64_t p = base + i;
            const int64_t o = base + written + ex;
            const double u = P.uv64[2 * p] * scale, v = P.uv64[2 * p + 1] * scale;
            const double X0 = P.X64[3 * p], X1 = P.X64[3 * p + 1], X2 = P.X64[3 * p + 2];
            P.lx64[2 * o] = u;
            P.lx64[2 * o + 1] = v;
            P.lX64[3 * o] = X0;
            P.lX64[3 * o + 1] = X1;
            P.lX64[3 * o + 2] = X2;
        }
        written += tot;
    }
    if (threadIdx.x == 0) {
        f.num_inliers = written;
        f.status = kLMPending;
        FrameResult &res = P.results[slot];
        for (int k = 0; k < 4; ++k) res.q[k] = sq[k];
        for (int k = 0; k < 3; ++k) res.t[k] = st[k];
    }
}

// ------------------------------------------------------------------ LM -----
__device__ __forceinline__ void kahan_add(float &s, float &c, float x) {
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// Block-wide FP64 sum of NV values per thread; every thread gets the result in
// out[] (shared). Uses 32*NV doubles of scratch.
template <int NV>
__device__ __forceinline__ void block_sum_d(double (&v)[NV], double *scratch, double *out) {
    static_assert(NV <= 32, "one value per lane after the warp reduction");
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // Warp reduce-scatter by recursive halving: at width h a lane trades the
    // half of its 2h partial sums that its partner (lane ^ h) keeps, so after
    // 16 + 8 + 4 + 2 + 1 exchanges lane k holds the warp's sum of value k.
    double a[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) a[k] = k < NV ? v[k] : 0.0;
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
        const bool upper = (lane & h) != 0;
#pragma unroll
        for (int k = 0; k < h; ++k) {
            const double keep = upper ? a[k + h] : a[k];
            const double give = upper ? a[k] : a[k + h];
            a[k] = keep + __shfl_xor_sync(0xffffffffu, give, h);
        }
    }
    if (lane < NV) scratch[w * NV + lane] = a[0];
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int q = 0; q < nw; ++q) s += scratch[q * NV + threadIdx.x];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

constexpr int kLMCluster = 8;  // CTAs cooperating on one frame's LM

constexpr int kLMSums = 28;  // cost + 21 J^T W J + 6 J^T W r
enum LMLoss : int32_t { kLossCauchy = 0, kLossTruncated = 1, kLossHuber = 2, kLossTrivial = 3 };

// One pass over inliers [i0, i1) at pose (q, t): the FP64 Cauchy cost
// (jaco.cuh:31-104) and, from the same FP64 residuals, the J^T W J lower
// triangle (jaco.cuh:173-200) and J^T W r (:202-209) accumulated in FP32 with
// Kahan compensation. The Jacobian uses the world coordinates of the
// reference's parameterisation (rotation post-multiplied, translation t + R dt).
// out[0] = cost, out[1..27] = accumulators (block totals).
__device__ void lm_pass(const Pools &P, int64_t base, int64_t i0, int64_t i1, const double *q, const double *t,
                        const double *cam, double inv_sq_thr, int loss, double thr, bool weighted,
                        double *scratch, double *out) {
    double R[9];
    quat_to_rotmat(q, R);
    const float r00 = (float)R[0], r01 = (float)R[1], r02 = (float)R[2], r10 = (float)R[3], r11 = (float)R[4],
                r12 = (float)R[5], r20 = (float)R[6], r21 = (float)R[7], r22 = (float)R[8];
    const float fx = (float)cam[0], fy = (float)cam[1];
    const float isq = (float)inv_sq_thr;
    double cost = 0.0;
    float Sv[27], Cc[27];
#pragma unroll
    for (int k = 0; k < 27; ++k) Sv[k] = Cc[k] = 0.0f;
#pragma unroll 2  // two points per thread in flight: the FP64 division and log1p chains overlap
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const int64_t o = base + i;
        const double X0d = P.lX64[3 * o], X1d = P.lX64[3 * o + 1], X2d = P.lX64[3 * o + 2];
        const double Z0 = R[0] * X0d + R[1] * X1d + R[2] * X2d + t[0];
        const double Z1 = R[3] * X0d + R[4] * X1d + R[5] * X2d + t[1];
        const double Z2 = R[6] * X0d + R[7] * X1d + R[8] * X2d + t[2];
        const bool valid = Z2 >= 0.0;
        const double inv_z = 1.0 / Z2;
        const double z0d = Z0 * inv_z, z1d = Z1 * inv_z;
        const double r0 = (cam[0] * z0d + cam[2]) - P.lx64[2 * o];
        const double r1 = (cam[1] * z1d + cam[3]) - P.lx64[2 * o + 1];
        const double r_squared = r0 * r0 + r1 * r1;
        // FP32 Jacobian from the FP64 projection and residual.
        const float iz = (float)inv_z, z0 = (float)z0d, z1 = (float)z1d;
        const float rx = (float)r0, ry = (float)r1;
        const float r2 = (float)r_squared;
        float wgt;
        double lc;
        if (loss == kLossCauchy) {  // CauchyLoss_cuda, robust_loss.cuh:24-38
            lc = log1p(r_squared * inv_sq_thr);
            wgt = fmaxf(isq / (1.0f + r2 * isq), FLT_MIN);
        } else {
            const double sq = thr * thr;
            if (loss == kLossTruncated) {  // TruncatedLoss_cuda, robust_loss.cuh:10-22
                lc = fmin(r_squared, sq);
                wgt = r_squared < sq ? 1.0f : 0.0f;
            } else if (loss == kLossHuber) {
                lc = r_squared <= sq ? r_squared : 2.0 * thr * sqrt(r_squared) - sq;
                wgt = r_squared <= sq ? 1.0f : (float)(thr / sqrt(r_squared));
            } else {
                lc = r_squared;
                wgt = 1.0f;
            }
        }
        if (weighted) {
            const double m = P.lw64[o];
            lc *= m;
            wgt *= (float)m;
        }
        cost += valid ? lc : 0.0;
        const float wv = valid ? wgt : 0.0f;
        const float a0 = fx * iz, a2 = -fx * z0 * iz;
        const float b1 = fy * iz, b2 = -fy * z1 * iz;
        const float dZ00 = a0 * r00 + a2 * r20, dZ01 = a0 * r01 + a2 * r21, dZ02 = a0 * r02 + a2 * r22;
        const float dZ10 = b1 * r10 + b2 * r20, dZ11 = b1 * r11 + b2 * r21, dZ12 = b1 * r12 + b2 * r22;
        const float d00 = wv * (dZ00 * dZ00 + dZ10 * dZ10);
        const float d10 = wv * (dZ01 * dZ00 + dZ11 * dZ10);
        const float d11 = wv * (dZ01 * dZ01 + dZ11 * dZ11);
        const float d20 = wv * (dZ02 * dZ00 + dZ12 * dZ10);
        const float d21 = wv * (dZ02 * dZ01 + dZ12 * dZ11);
        const float d22 = wv * (dZ02 * dZ02 + dZ12 * dZ12);
        const float X0 = (float)X0d, X1 = (float)X1d, X2 = (float)X2d;
        const float wx = wv * rx, wy = wv * ry;
        const float v[27] = {
            X2 * (X2 * d11 - X1 * d21) + X1 * (X1 * d22 - X2 * d21),
            -X2 * (X2 * d10 - X0 * d21) - X1 * (X0 * d22 - X2 * d20),
            X1 * (X0 * d21 - X1 * d20) - X2 * (X0 * d11 - X1 * d10),
            X1 * d20 - X2 * d10,
            X1 * d21 - X2 * d11,
            X1 * d22 - X2 * d21,
            X2 * (X2 * d00 - X0 * d20) + X0 * (X0 * d22 - X2 * d20),
            -X2 * (X1 * d00 - X0 * d10) - X0 * (X0 * d21 - X1 * d20),
            X2 * d00 - X0 * d20,
            X2 * d10 - X0 * d21,
            X2 * d20 - X0 * d22,
            X1 * (X1 * d00 - X0 * d10) + X0 * (X0 * d11 - X1 * d10),
            X0 * d10 - X1 * d00,
            X0 * d11 - X1 * d10,
            X0 * d21 - X1 * d20,
            d00, d10, d20, d11, d21, d22,
            wx * (X1 * dZ02 - X2 * dZ01) + wy * (X1 * dZ12 - X2 * dZ11),
            -wx * (X0 * dZ02 - X2 * dZ00) - wy * (X0 * dZ12 - X2 * dZ10),
            wx * (X0 * dZ01 - X1 * dZ00) + wy * (X0 * dZ11 - X1 * dZ10),
            dZ00 * wx + dZ10 * wy,
            dZ01 * wx + dZ11 * wy,
            dZ02 * wx + dZ12 * wy};
#pragma unroll
        for (int k = 0; k < 27; ++k) kahan_add(Sv[k], Cc[k], v[k]);
    }
    double dv[kLMSums];
    dv[0] = cost;
#pragma unroll
    for (int k = 0; k < 27; ++k) dv[1 + k] = (double)Sv[k] - (double)Cc[k];
    block_sum_d<kLMSums>(dv, scratch, out);
}

// 6x6 Cholesky solve of the damped normal equations (lm_utils.cuh:14-100),
// non-positive pivots replaced by 1e-15 as there, with reciprocal pivots.
__device__ __forceinline__ void cholesky_solve6(const double *A, const double *b, double *x) {
    double L[36], inv[6], y[6];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j <= i; ++j) {
            double sum = 0.0;
            for (int k = 0; k < j; ++k) sum += L[i * 6 + k] * L[j * 6 + k];
            if (i == j) {
                double val = A[i * 6 + i] - sum;
                if (val <= 0.0) val = 1e-15;
                L[i * 6 + i] = sqrt(val);
                inv[i] = 1.0 / L[i * 6 + i];
            } else {
                L[i * 6 + j] = (A[i * 6 + j] - sum) * inv[j];
            }
        }
    for (int i = 0; i < 6; ++i) {
        double sum = 0.0;
        for (int j = 0; j < i; ++j) sum += L[i * 6 + j] * y[j];
        y[i] = (b[i] - sum) * inv[i];
    }
    for (int i = 5; i >= 0; --i) {
        double sum = 0.0;
        for (int j = i + 1; j < 6; ++j) sum += L[j * 6 + i] * x[j];
        x[i] = (y[i] - sum) * inv[i];
    }
}

// Levenberg-Marquardt with the control flow of lm.cuh:15-171 -- damping, the
// accept rule, the lambda schedule, the removal of damping after a rejected
// step, and both stop tests -- one frame per cluster of CL CTAs, each owning a
// slice of the inliers. Every candidate pose gets one fused pass (cost and, for
// the case it is accepted, the normal equations at it), so an iteration costs
// one pass and two cluster barriers. Sums cross the block and cluster in FP64 in
// a fixed order; the solve, the step and the acceptance test are FP64.
template <int CL>
__device__ __forceinline__ void lm_frame(const Pools &P, int slot) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    __shared__ double scratch[32 * kLMSums];
    __shared__ double part[kLMSums];  // this CTA's pass totals
    __shared__ double tot[kLMSums];   // rank 0: cluster totals
    __shared__ double J[36], g[6], Jc[28], q[4], t[3], qn[4], tn[3];
    __shared__ double cost, lambda;
    __shared__ int brk, recompute, iters, invalid;
    __shared__ double pq[4], pt[3];  // the pose every CTA evaluates next
    __shared__ int pbrk;
    const int rank = (int)cluster.block_rank();
    FrameDev &f = P.frames[slot];
    FrameResult &res = P.results[slot];
    const int64_t base = f.blk_off * kSub;
    const int64_t n = f.num_inliers;
    const int64_t i0 = n * rank / CL, i1 = n * (rank + 1) / CL;
    const double cam[4] = {f.lm_cam[0], f.lm_cam[1], f.lm_cam[2], f.lm_cam[3]};
    const double inv_sq_thr = f.lm_inv_sq_thr;
    const int64_t max_it = f.skip_refine ? 0 : f.lm_max_iter;
    // Read once: every barrier of the loop would reload them from the record.
    const double grad_tol = f.lm_grad_tol, step_tol = f.lm_step_tol, min_lambda = f.lm_min_lambda,
                 max_lambda = f.lm_max_lambda, thr = f.lm_thr;
    const int loss = f.lm_loss;
    const bool weighted = f.lm_weighted != 0;

    auto cluster_totals = [&]() {  // after lm_pass: every CTA's part -> rank 0's tot
        cluster.sync();
        if (rank == 0 && threadIdx.x < kLMSums) {
            double acc = 0.0;
            for (int r = 0; r < CL; ++r) acc += cluster.map_shared_rank(part, r)[threadIdx.x];
            tot[threadIdx.x] = acc;
        }
        __syncthreads();
    };

    if (threadIdx.x == 0) {
        for (int k = 0; k < 4; ++k) pq[k] = res.q[k];
        for (int k = 0; k < 3; ++k) pt[k] = res.t[k];
    }
    __syncthreads();
    if (max_it > 0)
        lm_pass(P, base, i0, i1, pq, pt, cam, inv_sq_thr, loss, thr, weighted, scratch, part);
    else if (threadIdx.x < kLMSums) part[threadIdx.x] = 0.0;
    __syncthreads();
    // One CTA: its pass totals are the frame's; a cluster sums its CTAs' in rank 0.
    const double *T = CL == 1 ? part : tot;
    if constexpr (CL > 1) cluster_totals();
    if (rank == 0 && threadIdx.x == 0) {
        for (int k = 0; k < 4; ++k) q[k] = pq[k];
        for (int k = 0; k < 3; ++k) t[k] = pt[k];
        cost = T[0];
        for (int k = 0; k < 27; ++k) Jc[k] = T[1 + k];
        Jc[27] = 0.0;
        lambda = f.lm_lambda0;
        recompute = 1;
        iters = 0;
        invalid = 0;
        res.lm_cost0 = cost;
    }
    for (int64_t it = 0; it < max_it; ++it) {
        if (rank == 0 && threadIdx.x == 0) {
            brk = 0;
            if (recompute) {
                // J from the pass at the current pose (lower triangle in the
                // reference's order); gradient test of lm.cuh:243-248.
                const int idx[21][2] = {{0, 0}, {1, 0}, {2, 0}, {3, 0}, {4, 0}, {5, 0}, {1, 1},
                                        {2, 1}, {3, 1}, {4, 1}, {5, 1}, {2, 2}, {3, 2}, {4, 2},
                                        {5, 2}, {3, 3}, {4, 3}, {5, 3}, {4, 4}, {5, 4}, {5, 5}};
                for (int k = 0; k < 36; ++k) J[k] = 0.0;
                for (int k = 0; k < 21; ++k) J[idx[k][0] * 6 + idx[k][1]] = Jc[k];
                double gn = 0.0;
                for (int k = 0; k < 6; ++k) {
                    g[k] = Jc[21 + k];
                    gn += g[k] * g[k];
                }
                if (sqrt(gn) < grad_tol) brk = 1;
            }
            for (int k = 0; k < 6; ++k) J[k * 7] += lambda;
            double x[6];
            cholesky_solve6(J, g, x);
            double sn = 0.0;
            for (int k = 0; k < 6; ++k) {
                x[k] = -1 * x[k];
                sn += x[k] * x[k];
            }
            if (sqrt(sn) < step_tol) brk = 1;
            quat_step_post(q, x, qn);  // jaco.cuh:288-299
            double dt[3];
            quat_rotate(q, x[3], x[4], x[5], dt);
            for (int k = 0; k < 3; ++k) tn[k] = t[k] + dt[k];
        }
        if constexpr (CL == 1) {
            // One CTA: the candidate pose and the stop flag are read in place;
            // the pass's own barriers order this thread's next writes to them.
            __syncthreads();
            if (brk) break;
            lm_pass(P, base, i0, i1, qn, tn, cam, inv_sq_thr, loss, thr, weighted, scratch, part);
        } else {
            cluster.sync();
            if (threadIdx.x == 0) {
                pbrk = cluster.map_shared_rank(&brk, 0)[0];
                const double *rq = cluster.map_shared_rank(qn, 0), *rt = cluster.map_shared_rank(tn, 0);
                for (int k = 0; k < 4; ++k) pq[k] = rq[k];
                for (int k = 0; k < 3; ++k) pt[k] = rt[k];
            }
            __syncthreads();
            if (pbrk) break;
            lm_pass(P, base, i0, i1, pq, pt, cam, inv_sq_thr, loss, thr, weighted, scratch, part);
            __syncthreads();
            cluster_totals();
        }
        if (rank == 0 && threadIdx.x == 0) {
            if (T[0] < cost) {
                for (int k = 0; k < 4; ++k) q[k] = qn[k];
                for (int k = 0; k < 3; ++k) t[k] = tn[k];
                lambda = fmax(min_lambda, lambda / 10);
                cost = T[0];
                for (int k = 0; k < 27; ++k) Jc[k] = T[1 + k];
                recompute = 1;
            } else {
                ++invalid;
                for (int k = 0; k < 6; ++k) J[k * 7] -= lambda;
                lambda = fmin(max_lambda, lambda * 10);
                recompute = 0;
            }
            ++iters;
        }
    }
    if (rank == 0 && threadIdx.x == 0) {
        for (int k = 0; k < 4; ++k) res.q[k] = q[k];
        for (int k = 0; k < 3; ++k) res.t[k] = t[k];
        res.lm_iters = iters;
        res.lm_invalid = invalid;
        res.lm_cost = cost;
        res.samples = f.samples_done;
        res.rounds = f.rounds_done;
        res.hypotheses = f.hyps_done;
        res.ransac_inliers = f.found ? f.best_count : 0;
        res.num_inliers = f.num_inliers;
        res.model_score = f.found ? f.best_score : DBL_MAX;
        res.best_sample = f.found ? f.best_sample : -1;
        res.best_sol = f.found ? f.best_sol : -1;
        res.steps = f.steps;
        res.rescored = f.rescored;
        res.overflow = f.overflow;
        res.status = kDone;
    }
    cluster.sync();  // no CTA leaves while rank 0 may still read its shared memory
    if (rank == 0 && threadIdx.x == 0) f.status = kDone;
}

// Frames with fewer inliers than Pools::lm_cluster_min run their LM on one CTA,
// larger ones on a cluster of kLMCluster CTAs. Beside RANSAC (the server's steps
// with many resident frames) throughput wins: one CTA up to kLMClusterMin. After
// a batch's last step, and in the server's steps with few frames, nothing else
// runs and the LM is the whole remaining time: clusters from kLMClusterMinTail.
constexpr int64_t kLMClusterMin = 10000;
constexpr int64_t kLMClusterMinTail = 3000;

__global__ void __launch_bounds__(kLMSmallThreads, 1) k_lm_small(Pools P) {
    const int slot = P.active[blockIdx.x];
    const FrameDev &f = P.frames[slot];
    if (f.status != kLMPending || f.num_inliers >= P.lm_cluster_min || f.lm_force_cluster) return;
    lm_frame<1>(P, slot);
}

__global__ void __cluster_dims__(kLMCluster, 1, 1) __launch_bounds__(kLMThreads, 2) k_lm(Pools P) {
    const int slot = P.active[blockIdx.x / kLMCluster];
    const FrameDev &f = P.frames[slot];
    // uniform across the cluster
    if (f.status != kLMPending || (f.num_inliers < P.lm_cluster_min && !f.lm_force_cluster)) return;
    lm_frame<kLMCluster>(P, slot);
}

// Host-stepped runs: close the step (stamp it) so that frames finished in it
// are taken by k_inliers right away.
__global__ void k_tick(Pools P) { P.counters[kCSteps] += 1; }

// Failure-path check: a wait on an mbarrier that nothing ever completes, with
// `polls` tries, must give up and leave the timeout bit for the host.
__global__ void k_debug_bounded_wait(unsigned long long *counters, uint32_t polls) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
        if (!mbar_wait(&bar, 0u, polls)) atomicOr(&counters[kCError], kErrTimeout);
    }
}

// Serving: the status of every active frame in one array (one copy to the host).
__global__ void k_gather_status(Pools P, int32_t *out) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < P.n_active; a += gridDim.x * blockDim.x)
        out[a] = P.frames[P.active[a]].status;
}

// ----------------------------------------------------------- loop control --
// Body tail of the captured batch loop: continue while any frame is still in
// RANSAC, with a step limit that turns a runaway loop into an error.
__global__ void k_loop_ctl(Pools P, cudaGraphConditionalHandle h, unsigned long long max_steps) {
    const unsigned long long steps = ++P.counters[kCSteps];
    unsigned v = P.counters[kCStillRansac] > 0 ? 1u : 0u;
    if (v && steps >= max_steps) {
        flag_error(P, kErrOverflow);
        v = 0u;
    }
    if (P.counters[kCError] & kErrTimeout) v = 0u;
    cudaGraphSetConditional(h, v);
}

// Frames of Q waiting for their data start RANSAC (their points are in the
// pool and prepared).
__global__ void k_activate(Pools Q) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < Q.n_active; a += gridDim.x * blockDim.x) {
        FrameDev &f = Q.frames[Q.active[a]];
        if (f.status == kPending) f.status = kRansac;
    }
}

// Restores the frames of a batch to their post-admission state.
__global__ void k_reset_frames(Pools P, const FrameDev *init) {
    const int a = blockIdx.x;
    if (a >= P.n_active) return;
    const int4 *src = reinterpret_cast<const int4 *>(init + a);
    int4 *dst = reinterpret_cast<int4 *>(P.frames + P.active[a]);
    for (int i = threadIdx.x; i < (int)(sizeof(FrameDev) / 16); i += blockDim.x) dst[i] = src[i];
    if (a == 0 && threadIdx.x < kCNum) P.counters[threadIdx.x] = 0;
}

// Correspondence ingestion: a table of byte ranges (tiles) copied into the
// pool, from device memory or from page-locked host memory read over the link
// (zero-copy). The table is an int64 tile count, a pad word, then the tiles.
struct IngestTile {
    const char *src;
    char *dst;
    int64_t bytes;  // a multiple of 8
};
constexpr int kIngestTileCap = 8192;           // tiles of one call, all tables together
constexpr size_t kIngestTileBytes = 256u << 10;

// Copies `bytes` (a multiple of 8) from src to dst with the threads of one
// CTA: 16-byte words four at a time when both ends allow it.
__device__ __forceinline__ void copy_block(const char *__restrict__ src, char *__restrict__ dst, int64_t bytes) {
    const int t = threadIdx.x, T = blockDim.x;
    if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
        const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
        uint4 *d4 = reinterpret_cast<uint4 *>(dst);
        const int64_t n4 = bytes / 16;
        int64_t i = t;
        for (; i + 3 * T < n4; i += 4 * T) {
            const uint4 a = s4[i], b = s4[i + T], c = s4[i + 2 * T], d = s4[i + 3 * T];
            d4[i] = a;
            d4[i + T] = b;
            d4[i + 2 * T] = c;
            d4[i + 3 * T] = d;
        }
        for (; i < n4; i += T) d4[i] = s4[i];
        if (t == 0 && (bytes & 15))
            reinterpret_cast<unsigned long long *>(dst)[bytes / 8 - 1] =
                reinterpret_cast<const unsigned long long *>(src)[bytes / 8 - 1];
    } else {
        const unsigned long long *s8 = reinterpret_cast<const unsigned long long *>(src);
        unsigned long long *d8 = reinterpret_cast<unsigned long long *>(dst);
        for (int64_t i = t; i < bytes / 8; i += T) d8[i] = s8[i];
    }
}

__global__ void __launch_bounds__(256) k_ingest(const int64_t *table) {
    const int64_t n = table[0];
    const IngestTile *tiles = reinterpret_cast<const IngestTile *>(table + 2);
    for (int64_t k = blockIdx.x; k < n; k += gridDim.x) {
        const IngestTile t = tiles[k];
        copy_block(t.src, t.dst, t.bytes);
    }
}

__global__ void k_set_shape(FrameDev *init, int n, int hr, int chunk_points) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    init[a].hr = hr;
    init[a].chunk_points = chunk_points;
}

// Admission: staged[a] -> frames[slots[a]] (one upload for a whole batch).
__global__ void k_admit_frames(FrameDev *frames, const FrameDev *staged, const int32_t *slots, int n) {
    const int a = blockIdx.x;
    if (a >= n) return;
    const int4 *src = reinterpret_cast<const int4 *>(staged + a);
    int4 *dst = reinterpret_cast<int4 *>(frames + slots[a]);
    for (int i = threadIdx.x; i < (int)(sizeof(FrameDev) / 16); i += blockDim.x) dst[i] = src[i];
}

// Results of the frames in slots[0..n) packed into one array (one download).
static_assert(sizeof(FrameResult) % 8 == 0, "FrameResult is copied in 8-byte words");
__global__ void k_gather_results(const FrameResult *results, const int32_t *slots, int n, FrameResult *out) {
    constexpr int W = (int)(sizeof(FrameResult) / 8);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)n * W;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int a = (int)(i / W), w = (int)(i % W);
        reinterpret_cast<unsigned long long *>(out + a)[w] =
            reinterpret_cast<const unsigned long long *>(results + slots[a])[w];
    }
}

// ------------------------------------------------- standalone entry points --
// get_inliers_mx (entry.cu:12-26) for a given pose over raw device arrays.
__global__ void k_pose_mask(const double *xn, const double *X, int64_t n, const double *qt,
                            double sq_thr, uint8_t *mask, unsigned long long *count) {
    double R[9];
    quat_to_rotmat(qt, R);
    const double t0 = qt[4], t1 = qt[5], t2 = qt[6];
    int c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double X0 = X[3 * i], X1 = X[3 * i + 1], X2 = X[3 * i + 2];
        const double Z0 = R[0] * X0 + R[1] * X1 + R[2] * X2 + t0;
        const double Z1 = R[3] * X0 + R[4] * X1 + R[5] * X2 + t1;
        const double Z2 = R[6] * X0 + R[7] * X1 + R[8] * X2 + t2;
        const double h0 = Z0 / Z2 - xn[2 * i], h1 = Z1 / Z2 - xn[2 * i + 1];
        const int in = (h0 * h0 + h1 * h1 < sq_thr && Z2 > 0.0) ? 1 : 0;
        mask[i] = (uint8_t)in;
        c += in;
    }
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// bundle_adjust_cuda input: the caller's (x, X) become the LM arrays as given
// (ba.cu:41-62), with FP32 copies centred on the AABB midpoint.
__global__ void k_lm_pack(Pools P) {
    const int slot = P.active[0];
    FrameDev &f = P.frames[slot];
    const int64_t base = f.blk_off * kSub;
    const double c0 = 0.5 * (ordered_to_dbl(f.bmin[0]) + ordered_to_dbl(f.bmax[0]));
    const double c1 = 0.5 * (ordered_to_dbl(f.bmin[1]) + ordered_to_dbl(f.bmax[1]));
    const double c2 = 0.5 * (ordered_to_dbl(f.bmin[2]) + ordered_to_dbl(f.bmax[2]));
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        f.centre[0] = c0;
        f.centre[1] = c1;
        f.centre[2] = c2;
        f.num_inliers = f.n;
    }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < f.n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = base + i;
        const double u = P.uv64[2 * p], v = P.uv64[2 * p + 1];
        const double X0 = P.X64[3 * p], X1 = P.X64[3 * p + 1], X2 = P.X64[3 * p + 2];
        P.lx64[2 * p] = u;
        P.lx64[2 * p + 1] = v;
        P.lX64[3 * p] = X0;
        P.lX64[3 * p + 1] = X1;
        P.lX64[3 * p + 2] = X2;
    }
}

// ------------------------------------------------------------ FP32 peak ----
// Independent packed-FMA chains: 8 FP32x2 accumulators per thread, each step
// 8 fma.rn.f32x2 (32 FLOP per thread per step). The store is conditional on a
// value that never occurs, so nothing is written but nothing is dead code.
__global__ void __launch_bounds__(256) k_fp32_peak(float *sink, int iters, float a, float b) {
    uint64_t acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = f2pack(a + k + threadIdx.x, b - k);
    const uint64_t m = f2pack(a, a), c = f2pack(b, b);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = f2fma(acc[k], m, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float lo, hi;
        f2unpack(acc[k], lo, hi);
        s += lo + hi;
    }
    if (s == -12345.678f) sink[threadIdx.x] = s;
}

// ------------------------------------------------------------- debug -------
// Per-hypothesis inlier counts decided in FP32 (same formula as k_score),
// with pairs whose FP32 r^2/tau^2 lies within 2^-10 of 1 (or whose depth is
// within 2^-20 of zero) re-decided with the FP64 reference formula.
__global__ void k_debug_counts(Pools P) {
    const int slot = P.active[0];
    const FrameDev &f = P.frames[slot];
    const int64_t base = f.blk_off * kSub;
    for (int h = blockIdx.x; h < f.hyp_count; h += gridDim.x) {
        const float *Q = P.hP32 + 12 * (f.hyp_base + h);
        const double *M = P.hP64 + 12 * (f.hyp_base + h);
        int cnt = 0;
        for (int64_t i = threadIdx.x; i < f.n; i += blockDim.x) {
            const float2 *blk = P.pts32 + (f.blk_off + i / kSub) * kBlockFloat2;
            const int j = (int)(i % kSub);
            const float X = blk[j].x, Y = blk[kSub + j].x, Z = blk[2 * kSub + j].x;
            const float NX = blk[3 * kSub + j].x, NY = blk[4 * kSub + j].x;
            const float z0 = fmaf(Q[0], X, fmaf(Q[1], Y, fmaf(Q[2], Z, Q[3])));
            const float z1 = fmaf(Q[4], X, fmaf(Q[5], Y, fmaf(Q[6], Z, Q[7])));
            const float z2 = fmaf(Q[8], X, fmaf(Q[9], Y, fmaf(Q[10], Z, Q[11])));
            const float inv = rcp_approx(z2);
            const float r0 = fmaf(z0, inv, NX), r1 = fmaf(z1, inv, NY);
            const float qv = fmaf(r0, r0, r1 * r1);
            int in;
            if (fabsf(qv - 1.0f) < (1.0f / 1024.0f) || fabsf(z2) < 1e-6f || !(qv == qv)) {
                const int64_t p = base + i;
                const double X0 = P.X64[3 * p], X1 = P.X64[3 * p + 1], X2 = P.X64[3 * p + 2];
                const double d0 = M[0] * X0 + M[1] * X1 + M[2] * X2 + M[3];
                const double d1 = M[4] * X0 + M[5] * X1 + M[6] * X2 + M[7];
                const double d2 = M[8] * X0 + M[9] * X1 + M[10] * X2 + M[11];
                const double iv = 1.0 / d2;
                const double e0 = d0 * iv - P.xn64[2 * p], e1 = d1 * iv - P.xn64[2 * p + 1];
                in = (e0 * e0 + e1 * e1 < f.sq_thr && d2 > 0.0) ? 1 : 0;
            } else {
                in = (qv < 1.0f && z2 > 0.0f) ? 1 : 0;
            }
            cnt += in;
        }
        cnt = warp_sum(cnt);
        __shared__ int sc[32];
        if ((threadIdx.x & 31) == 0) sc[threadIdx.x >> 5] = cnt;
        __syncthreads();
        if (threadIdx.x == 0) {
            int s = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sc[k];
            P.dbg_counts[h] = s;
        }
        __syncthreads();
    }
}

}  // namespace tbr
