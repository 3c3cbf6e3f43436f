// Host engine and C ABI of libtbr.so (see include/tbr.h).
//
// One Engine per tbr_context: a CUDA stream, a device workspace carved once
// from one allocation (points, staging blocks, hypotheses, candidates, LM
// arrays), pinned host staging, and the step launcher. The reference allocates
// and frees every buffer per call (turbo_ransac.cu:36-112, 272-286; ba.cu:41-62)
// and synchronises the whole device 4 times per round; here nothing is
// allocated per call and a round needs no host round-trip.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/tbr.h"
#include "tbr_kernels.cuh"

namespace tbr {

thread_local std::string g_last_error;

static tbr_status fail(tbr_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

#define TBR_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(TBR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));         \
    } while (0)

// First-fit allocator over staging blocks, with coalescing on free.
class BlockAllocator {
   public:
    void reset(int64_t cap) {
        free_.clear();
        if (cap > 0) free_[0] = cap;
        cap_ = cap;
        used_ = 0;
    }
    int64_t alloc(int64_t n) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                const int64_t off = it->first, sz = it->second;
                free_.erase(it);
                if (sz > n) free_[off + n] = sz - n;
                used_ += n;
                return off;
            }
        }
        return -1;
    }
    void release(int64_t off, int64_t n) {
        used_ -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    int64_t used() const { return used_; }
    int64_t capacity() const { return cap_; }

   private:
    std::map<int64_t, int64_t> free_;
    int64_t cap_ = 0, used_ = 0;
};

struct FrameHost {
    const double *uv;
    const double *xyz;
    int64_t n;
    double K[4];
    uint64_t seed;
    double max_reproj_error;
    const int32_t *replay;  // host
    int64_t replay_count;
};

struct RunOptions {
    int64_t B = 1000;
    int64_t max_total = 100000;
    int64_t min_samples = 0;
    int64_t force_samples = 0;
    int prosac = 0;
    double prosac_TN = 100000.0;
    double success_prob = 0.9999;
    double trials_mult = 3.0;
    int skip_refine = 0;
    int quirk = 0;
    // Scoring shape: hr = 1 is the tensor-core kernel (32 hypotheses per block,
    // pp = kTcPP), the default; hr = 2, 4, 6, 8 with pp = 2 or 4 the FP32 kernels.
    int hr = 1;
    int pp = kTcPP;
    int chunk_points = 0;
    int max_rounds_step = 0;
    // LM (compat: default BundleOptions_cuda with loss_scale = 1/f)
    int64_t lm_max_iter = 100;
    double lm_loss_scale_px = 1.0;  // loss scale in pixels (multiplied by 1/f)
    double lm_grad_tol = 1e-10, lm_step_tol = 1e-8, lm_lambda0 = 1e-3, lm_min_lambda = 1e-10,
           lm_max_lambda = 1e10;
};

static RunOptions make_run_options(const tbr_ransac_options *ro, const tbr_bundle_options *bo,
                                   const tbr_ext_options *ext) {
    RunOptions o;
    if (ro) o.B = (int64_t)ro->max_iterations;
    const bool honor = ext && ext->honor_options;
    if (ext) {
        o.skip_refine = ext->skip_refine;
        o.quirk = ext->stop_rule_x86_quirk;
        o.force_samples = ext->force_samples;
        if (ext->max_total_samples > 0) o.max_total = ext->max_total_samples;
        // An FP32 shape is asked for by either of its fields; the other takes
        // its FP32 default (hr 4, pp 2). points_per_iter = kTcPP asks for the
        // tensor-core kernel whatever hyp_per_thread says.
        const int hpt = ext->hyp_per_thread, ppi = ext->points_per_iter;
        const bool fp32_hr = hpt == 2 || hpt == 4 || hpt == 6 || hpt == 8;
        const bool fp32_pp = ppi == 2 || ppi == 4;
        if (ppi == kTcPP) {
            o.hr = 1;
            o.pp = kTcPP;
        } else if (fp32_hr || fp32_pp) {
            o.hr = fp32_hr ? hpt : 4;
            o.pp = fp32_pp ? ppi : 2;
        }
        o.chunk_points = ext->chunk_points;
    }
    if (honor && ro) {
        o.success_prob = ro->success_prob;
        o.trials_mult = ro->dyn_num_trials_mult;
        o.min_samples = (int64_t)ro->min_iterations;
        o.prosac = ro->progressive_sampling ? 1 : 0;
        if (ro->max_prosac_iterations > 0) o.prosac_TN = (double)ro->max_prosac_iterations;
    }
    if (honor && bo) {
        o.lm_max_iter = (int64_t)bo->max_iterations;
        o.lm_loss_scale_px = bo->loss_scale;
        o.lm_grad_tol = bo->gradient_tol;
        o.lm_step_tol = bo->step_tol;
        o.lm_lambda0 = bo->initial_lambda;
        o.lm_min_lambda = bo->min_lambda;
        o.lm_max_lambda = bo->max_lambda;
    }
    return o;
}

class Engine {
   public:
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 148;
    Pools P{};            // device pointers (host copy)
    int max_frames = 0;
    int64_t max_blocks = 0;
    void *d_base = nullptr;
    size_t d_bytes = 0;
    BlockAllocator blocks;
    std::vector<int> free_slots;
    // pinned host staging
    void *h_stage = nullptr;
    size_t h_stage_bytes = 0;
    unsigned long long *h_counters = nullptr;
    FrameResult *h_results = nullptr;  // pinned: one call's packed results
    int32_t *d_active = nullptr;
    FrameDev *d_admit = nullptr;         // admission staging (device side)
    FrameResult *d_res_stage = nullptr;  // packed results of one download
    char *d_ingest = nullptr;            // ingestion tables of one admission (k_ingest)
    cudaEvent_t ev_ingest = nullptr;     // the caller's stream, waited on before ingestion
    int32_t *d_res_slots = nullptr;      // slot list of that download
    int32_t *d_replay = nullptr;
    int64_t d_replay_cap = 0;
    int score_grid[6] = {0, 0, 0, 0, 0, 0};  // (HP, PP) = (1,4), (2,2), (2,4), (4,2), (3,2), (3,4)
    int rescore_grid = 0, p3p_grid = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t stream2 = nullptr;             // late frames' ingestion in captured graphs; serving refinement
    cudaStream_t stream3 = nullptr;             // cluster LM beside the one-CTA LM
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_lm_fork = nullptr, ev_lm_join = nullptr;
    void *d_stage_alias = nullptr;              // device address of the pinned staging buffer
    cudaEvent_t ev_done = nullptr;              // a submitted batch's downloads have landed
    cudaStream_t stream_out = nullptr;          // inlier masks of a collected batch
    // Ingestion of the first part of a host batch runs on stream_in, beside
    // whatever the context stream still runs (it writes only the new frames'
    // blocks, from tables in d_ingest_first); the context stream waits on
    // ev_in before it prepares those frames.
    cudaStream_t stream_in = nullptr;
    cudaEvent_t ev_in = nullptr;
    char *d_ingest_first = nullptr;
    std::mutex mu;  // one call at a time per context

    // Per-call buffers: h_stage (with its size and device alias),
    // d_ingest_first, h_counters, h_results, ev0, ev1 and ev_done above are
    // the bound set;
    // `spare` holds the other one. Submitted batches use the two sets in turn
    // (next_set), so that one can be staged while the other's copies and
    // downloads are still queued; owner[k] is the ticket whose queued work
    // uses set k (nullptr: none).
    struct CallBuffers {
        void *h_stage = nullptr;
        size_t h_stage_bytes = 0;
        void *d_stage_alias = nullptr;
        char *d_ingest_first = nullptr;
        unsigned long long *h_counters = nullptr;
        FrameResult *h_results = nullptr;
        cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_done = nullptr;
    };
    CallBuffers spare;
    int bound = 0, next_set = 0;
    ::tbr_ticket *owner[2] = {nullptr, nullptr};
    void bind_set(int k) {
        if (k == bound) return;
        std::swap(h_stage, spare.h_stage);
        std::swap(h_stage_bytes, spare.h_stage_bytes);
        std::swap(d_stage_alias, spare.d_stage_alias);
        std::swap(d_ingest_first, spare.d_ingest_first);
        std::swap(h_counters, spare.h_counters);
        std::swap(h_results, spare.h_results);
        std::swap(ev0, spare.ev0);
        std::swap(ev1, spare.ev1);
        std::swap(ev_done, spare.ev_done);
        bound = k;
    }

    ~Engine() {
        if (stream) cudaStreamSynchronize(stream);
        if (stream_in) cudaStreamSynchronize(stream_in);
        for (auto &g : graph_cache) cudaGraphExecDestroy(g.exec);
        if (d_base) cudaFree(d_base);
        if (h_stage) cudaFreeHost(h_stage);
        if (h_counters) cudaFreeHost(h_counters);
        if (h_results) cudaFreeHost(h_results);
        if (d_replay) cudaFree(d_replay);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (ev_lm_fork) cudaEventDestroy(ev_lm_fork);
        if (ev_lm_join) cudaEventDestroy(ev_lm_join);
        if (stream3) cudaStreamDestroy(stream3);
        if (ev_ingest) cudaEventDestroy(ev_ingest);
        if (ev_done) cudaEventDestroy(ev_done);
        if (stream_out) cudaStreamDestroy(stream_out);
        if (stream_in) cudaStreamDestroy(stream_in);
        if (ev_in) cudaEventDestroy(ev_in);
        if (spare.h_stage) cudaFreeHost(spare.h_stage);
        if (spare.h_counters) cudaFreeHost(spare.h_counters);
        if (spare.h_results) cudaFreeHost(spare.h_results);
        if (spare.ev0) cudaEventDestroy(spare.ev0);
        if (spare.ev1) cudaEventDestroy(spare.ev1);
        if (spare.ev_done) cudaEventDestroy(spare.ev_done);
        if (stream2) cudaStreamDestroy(stream2);
        if (stream) cudaStreamDestroy(stream);
    }

    tbr_status init(int dev, uint64_t budget, int frames_cap = kMaxActive) {
        device = dev;
        TBR_CUDA(cudaSetDevice(dev));
        TBR_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
        TBR_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        TBR_CUDA(cudaEventCreate(&ev0));
        TBR_CUDA(cudaEventCreate(&ev1));
        TBR_CUDA(cudaStreamCreateWithFlags(&stream2, cudaStreamNonBlocking));
        TBR_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        TBR_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
        TBR_CUDA(cudaStreamCreateWithFlags(&stream3, cudaStreamNonBlocking));
        TBR_CUDA(cudaEventCreateWithFlags(&ev_lm_fork, cudaEventDisableTiming));
        TBR_CUDA(cudaEventCreateWithFlags(&ev_lm_join, cudaEventDisableTiming));
        TBR_CUDA(cudaEventCreateWithFlags(&ev_ingest, cudaEventDisableTiming));
        TBR_CUDA(cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
        TBR_CUDA(cudaStreamCreateWithFlags(&stream_out, cudaStreamNonBlocking));
        TBR_CUDA(cudaStreamCreateWithFlags(&stream_in, cudaStreamNonBlocking));
        TBR_CUDA(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
        TBR_CUDA(cudaEventCreate(&spare.ev0));
        TBR_CUDA(cudaEventCreate(&spare.ev1));
        TBR_CUDA(cudaEventCreateWithFlags(&spare.ev_done, cudaEventDisableTiming));
        if (budget == 0) budget = 1ull << 30;
        max_frames = std::min(frames_cap, kMaxActive);
        // Split: 30 % hypotheses, the rest points, after the per-frame state.
        const size_t per_frame = 2 * (sizeof(FrameDev) + sizeof(FrameResult)) + sizeof(int32_t) + 64;
        P.cand_cap = std::max<int64_t>(16384, (int64_t)max_frames * 256);
        const size_t per_cand = 4 + 8 + 8 + 4 + (size_t)kMaxRChunks * 12;
        const size_t fixed = (size_t)max_frames * per_frame + (size_t)P.cand_cap * per_cand +
                             3 * (kMaxActive + 1) * 8 + 4096 * 8;
        if (budget < fixed + (64ull << 20)) return fail(TBR_ERR_INVALID_ARG, "workspace too small");
        const size_t rest = budget - fixed;
        const size_t per_hyp = 96 + 48 + 8 + 4 + 4 * 32 + 4;
        P.max_hyps = (int64_t)(rest * 0.3 / per_hyp);
        P.max_hyps = std::max<int64_t>(P.max_hyps, 4096);
        P.max_parts = P.max_hyps * 32;
        P.max_hb = P.max_hyps / 32 + kMaxActive;
        const size_t per_block = (size_t)kSub * (16 + 24 + 16 + 1 + 16 + 24 + 8 + 8) + kBlockBytes;
        max_blocks = (int64_t)((rest - (size_t)(P.max_hyps * per_hyp) - P.max_hb * 4) / per_block) - 1;
        if (max_blocks < 64) return fail(TBR_ERR_INVALID_ARG, "workspace too small for points");
        // One allocation, carved with 256-byte alignment.
        std::vector<std::pair<void **, size_t>> parts;
        const int64_t np = max_blocks * kSub;
        auto add = [&](void **p, size_t bytes) { parts.push_back({p, bytes}); };
        add((void **)&P.frames, sizeof(FrameDev) * max_frames);
        add((void **)&P.results, sizeof(FrameResult) * max_frames);
        add((void **)&d_active, sizeof(int32_t) * kMaxActive);
        add((void **)&d_admit, sizeof(FrameDev) * kMaxActive);
        add((void **)&d_res_stage, sizeof(FrameResult) * kMaxActive);
        add((void **)&d_ingest, kIngestTableBytes);
        add((void **)&d_ingest_first, kIngestTableBytes);
        add((void **)&spare.d_ingest_first, kIngestTableBytes);
        add((void **)&d_res_slots, sizeof(int32_t) * kMaxActive);
        add((void **)&P.uv64, 16 * np);
        add((void **)&P.X64, 24 * np);
        add((void **)&P.xn64, 16 * np);
        add((void **)&P.mask, np);
        add((void **)&P.lx64, 16 * np);
        add((void **)&P.lX64, 24 * np);
        add((void **)&P.lw64, 8 * np);
        add((void **)&P.prosac64, 8 * np);
        add((void **)&P.pts32, (size_t)kBlockBytes * max_blocks);
        add((void **)&P.sample_prefix, 8 * (kMaxActive + 1));
        add((void **)&P.item_prefix, 8 * (kMaxActive + 1));
        add((void **)&P.ritem_prefix, 8 * (kMaxActive + 1));
        add((void **)&P.hP64, 96 * P.max_hyps);
        add((void **)&P.hP32, 48 * P.max_hyps);
        add((void **)&P.hId, 8 * P.max_hyps);
        add((void **)&P.hS32, 4 * P.max_hyps);
        add((void **)&P.part, 4 * P.max_parts);
        add((void **)&P.hb_arrive, 4 * P.max_hb);
        add((void **)&P.cHyp, 4 * (size_t)P.cand_cap);
        add((void **)&P.cS64, 8 * (size_t)P.cand_cap);
        add((void **)&P.cCnt, 8 * (size_t)P.cand_cap);
        add((void **)&P.cpS, 8 * (size_t)P.cand_cap * kMaxRChunks);
        add((void **)&P.cpC, 4 * (size_t)P.cand_cap * kMaxRChunks);
        add((void **)&P.c_arrive, 4 * (size_t)P.cand_cap);
        add((void **)&P.counters, 8 * kCNum);
        add((void **)&P.dbg_counts, 8 * P.max_hyps);
        size_t total = 0;
        for (auto &p : parts) total += (p.second + 255) & ~size_t(255);
        TBR_CUDA(cudaMalloc(&d_base, total));
        d_bytes = total;
        char *cur = (char *)d_base;
        for (auto &p : parts) {
            *p.first = cur;
            cur += (p.second + 255) & ~size_t(255);
        }
        P.active = d_active;
        P.num_sms = num_sms;
        P.lm_cluster_min = kLMClusterMin;
        TBR_CUDA(cudaMemsetAsync(P.frames, 0, sizeof(FrameDev) * max_frames, stream));
        TBR_CUDA(cudaMallocHost(&h_counters, 8 * kCNum));
        TBR_CUDA(cudaMallocHost(&h_results, sizeof(FrameResult) * kMaxActive));
        TBR_CUDA(cudaMallocHost(&spare.h_counters, 8 * kCNum));
        TBR_CUDA(cudaMallocHost(&spare.h_results, sizeof(FrameResult) * kMaxActive));
        blocks.reset(max_blocks);
        for (int i = max_frames - 1; i >= 0; --i) free_slots.push_back(i);
        int occ = 0;
        const void *sk[6] = {(const void *)k_score<1, 4>, (const void *)k_score<2, 2>, (const void *)k_score<2, 4>,
                             (const void *)k_score<4, 2>, (const void *)k_score<3, 2>, (const void *)k_score<3, 4>};
        for (int v = 0; v < 6; ++v) {
            TBR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sk[v], kScoreWarps * 32, 0));
            score_grid[v] = num_sms * std::max(occ, 1);
        }
        TBR_CUDA(cudaFuncSetAttribute(k_score_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
        TBR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rescore, 256, 0));
        rescore_grid = num_sms * std::max(occ, 1);
        p3p_grid = num_sms * 8;
        TBR_CUDA(cudaStreamSynchronize(stream));
        return TBR_OK;
    }

    tbr_status ensure_stage(size_t bytes) {
        if (bytes <= h_stage_bytes) return TBR_OK;
        if (h_stage) {
            TBR_CUDA(cudaStreamSynchronize(stream));
            cudaFreeHost(h_stage);
            h_stage = nullptr;
        }
        size_t nb = std::max(bytes, h_stage_bytes * 2);
        TBR_CUDA(cudaMallocHost(&h_stage, nb));
        h_stage_bytes = nb;
        d_stage_alias = nullptr;
        if (cudaHostGetDevicePointer(&d_stage_alias, h_stage, 0) != cudaSuccess) {
            cudaGetLastError();
            d_stage_alias = nullptr;
        }
        return TBR_OK;
    }

    tbr_status ensure_replay(int64_t count) {
        if (count <= d_replay_cap) return TBR_OK;
        if (d_replay) {
            TBR_CUDA(cudaStreamSynchronize(stream));
            cudaFree(d_replay);
            d_replay = nullptr;
        }
        TBR_CUDA(cudaMalloc(&d_replay, sizeof(int32_t) * 3 * count));
        d_replay_cap = count;
        return TBR_OK;
    }

    // Builds the device state of one frame (no device traffic).
    FrameDev make_frame(const FrameHost &fh, int64_t blk_off, const RunOptions &o,
                        const int32_t *d_rep) const {
        FrameDev f;
        std::memset(&f, 0, sizeof(f));
        f.n = fh.n;
        f.blk_off = blk_off;
        f.n_blocks = (int32_t)((fh.n + kSub - 1) / kSub);
        f.status = kRansac;
        f.seed = fh.seed;
        f.replay = d_rep;
        f.replay_count = fh.replay_count;
        for (int k = 0; k < 4; ++k) f.K[k] = fh.K[k];
        f.focal = 0.5 * (fh.K[0] + fh.K[1]);          // Camera_cuda::focal, camera.cuh:64-67
        f.tau = fh.max_reproj_error / f.focal;        // entry.cu:48-49
        f.sq_thr = f.tau * f.tau;                     // turbo_ransac.cu:34
        for (int k = 0; k < 3; ++k) {
            f.bmin[k] = ~0ull;
            f.bmax[k] = 0ull;
        }
        f.B = o.B;
        f.max_total = o.max_total;
        f.min_samples = o.min_samples;
        f.prosac = o.prosac;
        f.prosac_TN = o.prosac_TN;
        f.force_samples = o.force_samples;
        f.log_missing = std::log(1.0 - o.success_prob);
        f.trials_mult = o.trials_mult;
        f.skip_refine = o.skip_refine;
        f.quirk = o.quirk;
        f.hr = o.hr;
        f.chunk_points = o.chunk_points;
        f.max_rounds_step = o.max_rounds_step;
        f.lm_max_iter = o.lm_max_iter;
        const double sc = 1.0 / f.focal;  // entry.cu:87,107-114: LM in pixel/f units
        for (int k = 0; k < 4; ++k) f.lm_cam[k] = fh.K[k] * sc;
        const double ls = o.lm_loss_scale_px / f.focal;  // entry.cu:122-123
        f.lm_inv_sq_thr = 1.0 / (ls * ls);
        f.lm_grad_tol = o.lm_grad_tol;
        f.lm_step_tol = o.lm_step_tol;
        f.lm_lambda0 = o.lm_lambda0;
        f.lm_min_lambda = o.lm_min_lambda;
        f.lm_max_lambda = o.lm_max_lambda;
        f.best_score = DBL_MAX;
        f.best_sample = -1;
        f.best_sol = -1;
        return f;
    }

    // Enqueue the step kernels for the active list of `Q`. With `prof`, every
    // kernel is bracketed by CUDA events on this stream.
    struct Profile {
        cudaEvent_t ev[2 * 12] = {};
        double ms[12] = {};
        int64_t launches[12] = {};
        bool armed = false;
    };
    static constexpr const char *kKernelNames[12] = {"k_plan", "k_sample_p3p", "k_score_plan", "k_score",
                                                     "k_select", "k_rescore_plan", "k_rescore", "k_finalize",
                                                     "k_inliers", "k_lm", "k_prep", "unused"};
    // Scoring kernel variant: HR hypotheses per lane = 2*HP, PP points per iteration.
    void launch_score(const Pools &Q, int hr, int pp, cudaStream_t st) {
        const int threads = kScoreWarps * 32;
        if (hr == 1) k_score_tc<<<4 * num_sms, kTcThreads, kTcSmem, st>>>(Q);  // (pp == kTcPP)
        else if (hr == 2) k_score<1, 4><<<score_grid[0], threads, 0, st>>>(Q);
        else if (hr == 8) k_score<4, 2><<<score_grid[3], threads, 0, st>>>(Q);
        else if (hr == 6 && pp == 4) k_score<3, 4><<<score_grid[5], threads, 0, st>>>(Q);
        else if (hr == 6) k_score<3, 2><<<score_grid[4], threads, 0, st>>>(Q);
        else if (pp == 4) k_score<2, 4><<<score_grid[2], threads, 0, st>>>(Q);
        else k_score<2, 2><<<score_grid[1], threads, 0, st>>>(Q);
    }
    int pp = kTcPP;  // points per iteration of the scoring kernel (kTcPP: the tensor-core kernel)

    // RANSAC part of a step (plan .. finalize).
    void launch_ransac(const Pools &Q, int n_active, int hr, cudaStream_t st, Profile *prof = nullptr) {
        auto beg = [&](int k) { if (prof) cudaEventRecord(prof->ev[2 * k], st); };
        auto end = [&](int k) { if (prof) { cudaEventRecord(prof->ev[2 * k + 1], st); prof->launches[k]++; } };
        beg(0); k_plan<<<1, kMaxActive, 0, st>>>(Q); end(0);
        beg(1); k_sample_p3p<<<p3p_grid, 128, 0, st>>>(Q); end(1);
        beg(2); k_score_plan<<<1, kMaxActive, 0, st>>>(Q); end(2);
        beg(3);
        launch_score(Q, hr, pp, st);
        end(3);
        beg(4); k_select<<<n_active, 1024, 0, st>>>(Q); end(4);  // a frame's ~4000 hypotheses: 1024 threads (6.51 ms a batch, 256: 6.59)
        beg(5); k_rescore_plan<<<1, kMaxActive, 0, st>>>(Q); end(5);
        beg(6); k_rescore<<<rescore_grid, 256, 0, st>>>(Q); end(6);
        beg(7); k_finalize<<<n_active, 256, 0, st>>>(Q); end(7);
    }
    // Refinement part: inliers + LM of frames whose RANSAC ended in an earlier step.
    void launch_refine(const Pools &Q, int n_active, cudaStream_t st, Profile *prof = nullptr) {
        auto beg = [&](int k) { if (prof) cudaEventRecord(prof->ev[2 * k], st); };
        auto end = [&](int k) { if (prof) { cudaEventRecord(prof->ev[2 * k + 1], st); prof->launches[k]++; } };
        beg(8); k_inliers<<<n_active, 1024, 0, st>>>(Q); end(8);
        beg(9);
        // The one-CTA and the cluster LM take disjoint frames (by inlier
        // count): they run side by side, so the branch lasts as long as the
        // slower of the two, not their sum.
        cudaEventRecord(ev_lm_fork, st);
        cudaStreamWaitEvent(stream3, ev_lm_fork, 0);
        k_lm<<<n_active * kLMCluster, kLMThreads, 0, stream3>>>(Q);
        k_lm_small<<<n_active, kLMSmallThreads, 0, st>>>(Q);
        cudaEventRecord(ev_lm_join, stream3);
        cudaStreamWaitEvent(st, ev_lm_join, 0);
        end(9);
    }
    // Host-stepped: RANSAC, close the step, refine what finished.
    void launch_step(const Pools &Q, int n_active, int hr, Profile *prof = nullptr) {
        launch_ransac(Q, n_active, hr, stream, prof);
        k_tick<<<1, 1, 0, stream>>>(Q);
        launch_refine(Q, n_active, stream, prof);
    }

    void launch_prep(const Pools &Q, int n_active, int64_t max_n, cudaStream_t st) {
        const int bx = (int)std::min<int64_t>(64, std::max<int64_t>(1, (max_n + 1023) / 1024));
        k_prep_bounds<<<dim3(bx, n_active), 256, 0, st>>>(Q);
        k_prep_pack<<<dim3(bx, n_active), 256, 0, st>>>(Q);
        k_prosac_table<<<n_active, 1024, 0, st>>>(Q);
    }
    void launch_prep(const Pools &Q, int n_active, int64_t max_n) { launch_prep(Q, n_active, max_n, stream); }
    void launch_prep(int n_active, int64_t max_n) { launch_prep(P, n_active, max_n, stream); }

    static constexpr size_t kIngestTableBytes = 64 * 32 + sizeof(IngestTile) * kIngestTileCap;
    static constexpr int kIngestGridHost = 16;  // CTAs of a zero-copy ingestion: the link saturates at 16, and
                                                // late frames are read beside the first engine step
    static constexpr int kIngestGridBeside = 8;  // ... of one that runs beside another batch's run: there the
                                                 // SMs it takes from that run cost more than link rate
                                                 // (measured: 37.0k frames/s end to end against 36.4k with 16)

    // Split admission of a graph: the active frames from n_first on arrive
    // during the first step (kPending; their ingestion table at d_ingest).
    struct Stagger {
        int n_first = 0;
        int64_t max_n_rest = 0;
    };
    static int prep_bx(int64_t max_n) { return (int)std::min<int64_t>(64, std::max<int64_t>(1, (max_n + 1023) / 1024)); }

    // The step loop as one graph: [reset ->] while (any frame in RANSAC)
    // { RANSAC step ; loop test } -> inliers + LM of every frame. A frame's LM
    // is latency-bound and each one-CTA LM fills an SM, so running it beside
    // RANSAC stretched the steps more than refining every frame at the end,
    // with the whole GPU and clusters from kLMClusterMinTail inliers, costs
    // (6.46 ms against 6.52 ms a batch of the batched workload).
    // With d_init, a reset node first restores the frames from d_init. With sg,
    // the first step runs before the loop, beside the ingestion and preparation
    // of the frames that arrive late, which start RANSAC in the second step.
    bool build_loop_graph(const Pools &Q, int n, int hr, const FrameDev *d_init, cudaGraph_t *graph_out,
                          cudaGraphExec_t *exec_out, const Stagger *sg = nullptr) {
        cudaGraph_t graph = nullptr;
        cudaGraphConditionalHandle h;
        bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess &&
                  cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        cudaGraphNode_t reset_node = nullptr, loop_node = nullptr;
        Pools Qc = Q;
        const FrameDev *init = d_init;
        if (ok && d_init) {
            cudaKernelNodeParams kp = {};
            void *args[2] = {(void *)&Qc, (void *)&init};
            kp.func = (void *)k_reset_frames;
            kp.gridDim = dim3(n);
            kp.blockDim = dim3(128);
            kp.kernelParams = args;
            ok = cudaGraphAddKernelNode(&reset_node, graph, nullptr, 0, &kp) == cudaSuccess;
        }
        if (ok && sg && !d_init) {
            cudaGraph_t pro = nullptr;
            ok = cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed) == cudaSuccess;
            if (ok) {
                Pools Qr = Q;
                Qr.active = Q.active + sg->n_first;
                Qr.n_active = n - sg->n_first;
                cudaEventRecord(ev_fork, stream);
                cudaStreamWaitEvent(stream2, ev_fork, 0);
                k_ingest<<<kIngestGridHost, 256, 0, stream2>>>((const int64_t *)d_ingest);
                launch_prep(Qr, Qr.n_active, sg->max_n_rest, stream2);
                launch_ransac(Q, n, hr, stream);
                cudaEventRecord(ev_join, stream2);
                cudaStreamWaitEvent(stream, ev_join, 0);
                k_activate<<<1, kMaxActive, 0, stream>>>(Qr);
                k_tick<<<1, 1, 0, stream>>>(Q);
                ok = cudaStreamEndCapture(stream, &pro) == cudaSuccess;
            }
            if (ok) ok = cudaGraphAddChildGraphNode(&reset_node, graph, nullptr, 0, pro) == cudaSuccess;
            if (pro) cudaGraphDestroy(pro);
        }
        cudaGraph_t body = nullptr;
        if (ok) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            ok = cudaGraphAddNode(&loop_node, graph, reset_node ? &reset_node : nullptr, reset_node ? 1 : 0, &cp) ==
                 cudaSuccess;
            body = cp.conditional.phGraph_out[0];
        }
        if (ok) {
            ok = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed) ==
                 cudaSuccess;
            if (ok) {
                launch_ransac(Q, n, hr, stream);
                k_loop_ctl<<<1, 1, 0, stream>>>(Q, h, 100000ull);
                ok = cudaStreamEndCapture(stream, &body) == cudaSuccess;
            }
        }
        if (ok) {
            cudaGraph_t tail = nullptr;
            ok = cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed) == cudaSuccess;
            if (ok) {
                Pools Qt = Q;  // nothing runs beside the refinement
                Qt.lm_cluster_min = kLMClusterMinTail;
                launch_refine(Qt, n, stream);
                ok = cudaStreamEndCapture(stream, &tail) == cudaSuccess;
            }
            cudaGraphNode_t tail_node;
            if (ok) ok = cudaGraphAddChildGraphNode(&tail_node, graph, &loop_node, 1, tail) == cudaSuccess;
            if (tail) cudaGraphDestroy(tail);
        }
        cudaGraphExec_t exec = nullptr;
        if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        if (!ok) {
            cudaGetLastError();
            if (graph) cudaGraphDestroy(graph);
            return false;
        }
        *exec_out = exec;
        if (graph_out) *graph_out = graph;
        else cudaGraphDestroy(graph);
        return true;
    }

    // Instantiated loop graphs of recent (frame count, scoring variant) shapes,
    // least recently used first.
    struct CachedGraph {
        int n, hr, pp, n_first, bx;  // n_first, bx: split admission (0, 0 without)
        cudaGraphExec_t exec;
    };
    std::vector<CachedGraph> graph_cache;
    static constexpr size_t kGraphCacheSize = 8;

    // Enqueues the run of the active frames of P (admitted and prepared) to
    // completion as one graph launch; the counters must be zero.
    tbr_status launch_graph(int na, int hr, const Stagger *sg = nullptr) {
        cudaGraphExec_t exec = nullptr;
        const int nf = sg ? sg->n_first : 0, bx = sg ? prep_bx(sg->max_n_rest) : 0;
        for (size_t i = 0; i < graph_cache.size(); ++i)
            if (graph_cache[i].n == na && graph_cache[i].hr == hr && graph_cache[i].pp == pp &&
                graph_cache[i].n_first == nf && graph_cache[i].bx == bx) {
                CachedGraph g = graph_cache[i];
                graph_cache.erase(graph_cache.begin() + i);
                graph_cache.push_back(g);
                exec = g.exec;
                break;
            }
        if (!exec) {
            Stagger s2;
            if (sg) {  // the graph's preparation grid is sized for bx, whatever the frames
                s2.n_first = nf;
                s2.max_n_rest = (int64_t)bx * 1024;
            }
            if (!build_loop_graph(P, na, hr, nullptr, nullptr, &exec, sg ? &s2 : nullptr))
                return fail(TBR_ERR_CUDA, "graph capture failed");
            if (graph_cache.size() >= kGraphCacheSize) {
                cudaGraphExecDestroy(graph_cache.front().exec);
                graph_cache.erase(graph_cache.begin());
            }
            graph_cache.push_back({na, hr, pp, nf, bx, exec});
        }
        TBR_CUDA(cudaGraphLaunch(exec, stream));
        return TBR_OK;
    }

    // Runs the active frames of `Q` to completion with one host check per step.
    tbr_status run(const Pools &Q, int na, int hr, int max_steps, int *steps_out, Profile *prof = nullptr) {
        int steps = 0;
        if (prof && !prof->armed) {
            for (auto &e : prof->ev) TBR_CUDA(cudaEventCreate(&e));
            prof->armed = true;
        }
        for (;;) {
            launch_step(Q, na, hr, prof);
            TBR_CUDA(cudaGetLastError());
            TBR_CUDA(cudaMemcpyAsync(h_counters, Q.counters, 8 * kCNum, cudaMemcpyDeviceToHost, stream));
            TBR_CUDA(cudaStreamSynchronize(stream));
            if (prof)
                for (int k = 0; k < 10; ++k) {
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, prof->ev[2 * k], prof->ev[2 * k + 1]);
                    prof->ms[k] += ms;
                }
            ++steps;
            if (h_counters[kCError] & kErrTimeout) return fail(TBR_ERR_TIMEOUT, "bounded device wait expired");
            if (h_counters[kCStillRansac] == 0) break;
            if (steps >= max_steps) return fail(TBR_ERR_INTERNAL, "step limit reached");
        }
        TBR_CUDA(cudaStreamSynchronize(stream));
        if (steps_out) *steps_out = steps;
        return TBR_OK;
    }
    tbr_status run(const std::vector<int> &slots, int hr, int max_steps, int *steps_out) {
        return run(P, (int)slots.size(), hr, max_steps, steps_out);
    }
};

// Host copies into pinned staging, split over threads when the batch is large
// (a single core's memcpy bandwidth is well below the link's).
struct CopyJob {
    void *dst;
    const void *src;
    size_t bytes;
};
static void parallel_copy(const std::vector<CopyJob> &jobs) {
    constexpr size_t kChunk = 1 << 20;
    size_t total = 0;
    for (auto &j : jobs) total += j.bytes;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int T = (int)std::min<size_t>(std::min(8u, hw), total / (4 * kChunk));
    if (T <= 1) {
        for (auto &j : jobs) std::memcpy(j.dst, j.src, j.bytes);
        return;
    }
    std::vector<CopyJob> pieces;
    for (auto &j : jobs)
        for (size_t o = 0; o < j.bytes; o += kChunk)
            pieces.push_back({(char *)j.dst + o, (const char *)j.src + o, std::min(kChunk, j.bytes - o)});
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t k; (k = next.fetch_add(1)) < pieces.size();)
            std::memcpy(pieces[k].dst, pieces[k].src, pieces[k].bytes);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < T; ++t) th.emplace_back(work);
    work();
    for (auto &x : th) x.join();
}

// Admission in two halves. stage_frames (host only) takes slots and point
// blocks and copies the frames into pinned staging; upload_staged enqueues the
// device side. Frames whose point blocks are adjacent in the pool form one run;
// the staging area mirrors the pool's layout inside a run, so a run costs one
// copy per array. The frame records go up as one array and are scattered by
// one kernel; after the upload d_active[0..n) holds the new slots.
struct StagedAdmission {
    struct Run {
        int64_t b0, b1;  // block range in the pool
        char *huv, *hxyz;
    };
    std::vector<int> slots;
    std::vector<FrameDev> devs;
    std::vector<Run> runs;
    std::vector<std::pair<size_t, size_t>> span;  // first and last frame of each run
    std::vector<CopyJob> jobs;                    // uv, xyz of frame i at 2i, 2i+1
    FrameDev *hd = nullptr;
    int32_t *ha = nullptr;
    int64_t max_n = 0;
};

static size_t stage_bytes(const std::vector<FrameHost> &fr) {
    auto r256 = [](size_t b) { return (b + 255) & ~size_t(255); };
    size_t stage = 0;
    for (auto &f : fr) {
        const size_t pts = (size_t)((f.n + kSub - 1) / kSub) * kSub;
        stage += r256(16 * pts) + r256(24 * pts);
    }
    return stage + r256(sizeof(FrameDev) * fr.size()) + r256(4 * fr.size()) + 256;
}

// `stage` holds at least stage_bytes(fr) bytes of pinned memory that no copy in
// flight reads. With copy = false the host copies are left in A.jobs.
static tbr_status stage_frames(Engine &E, const std::vector<FrameHost> &fr, const RunOptions &o, char *stage,
                               StagedAdmission &A, bool copy = true, bool host_points = true) {
    if ((int)fr.size() > (int)E.free_slots.size()) return fail(TBR_ERR_CAPACITY, "too many frames for the context");
    auto r256 = [](size_t b) { return (b + 255) & ~size_t(255); };
    int64_t replay_total = 0;
    for (auto &f : fr) replay_total += f.replay ? f.replay_count : 0;
    if (replay_total) {
        tbr_status st = E.ensure_replay(replay_total);
        if (st) return st;
    }
    A = StagedAdmission();
    std::vector<int64_t> offs;
    int64_t rep_off = 0;
    for (auto &f : fr) {
        const int64_t nb = (f.n + kSub - 1) / kSub;
        const int64_t off = E.blocks.alloc(nb);
        if (off < 0) {
            for (size_t i = 0; i < A.slots.size(); ++i) E.blocks.release(A.devs[i].blk_off, A.devs[i].n_blocks);
            for (int s : A.slots) E.free_slots.push_back(s);
            A.slots.clear();
            return fail(TBR_ERR_OOM, "point workspace exhausted");
        }
        const int slot = E.free_slots.back();
        E.free_slots.pop_back();
        A.slots.push_back(slot);
        offs.push_back(off);
        const int32_t *d_rep = nullptr;
        if (f.replay) {
            d_rep = E.d_replay + 3 * rep_off;
            TBR_CUDA(cudaMemcpyAsync((void *)d_rep, f.replay, 12 * f.replay_count, cudaMemcpyHostToDevice, E.stream));
            rep_off += f.replay_count;
        }
        A.devs.push_back(E.make_frame(f, off, o, d_rep));
        A.max_n = std::max(A.max_n, f.n);
    }
    if (!host_points) {  // records only: the points come from device memory
        auto r256 = [](size_t b) { return (b + 255) & ~size_t(255); };
        A.hd = (FrameDev *)stage;
        A.ha = (int32_t *)(stage + r256(sizeof(FrameDev) * fr.size()));
        for (size_t i = 0; i < fr.size(); ++i) {
            A.hd[i] = A.devs[i];
            A.ha[i] = A.slots[i];
        }
        return TBR_OK;
    }
    // Runs of adjacent frames.
    auto &span = A.span;
    for (size_t i = 0; i < fr.size(); ++i) {
        const int64_t nb = A.devs[i].n_blocks;
        if (!A.runs.empty() && A.runs.back().b1 == offs[i]) {
            A.runs.back().b1 += nb;
            span.back().second = i;
        } else {
            A.runs.push_back({offs[i], offs[i] + nb, nullptr, nullptr});
            span.push_back({i, i});
        }
    }
    char *h = stage;
    auto &jobs = A.jobs;
    for (size_t r = 0; r < A.runs.size(); ++r) {
        auto &run = A.runs[r];
        const size_t pts = (size_t)(run.b1 - run.b0) * kSub;
        run.huv = h;
        h += r256(16 * pts);
        run.hxyz = h;
        h += r256(24 * pts);
        for (size_t i = span[r].first; i <= span[r].second; ++i) {
            const size_t p = (size_t)(offs[i] - run.b0) * kSub;
            jobs.push_back({run.huv + 16 * p, fr[i].uv, 16 * (size_t)fr[i].n});
            jobs.push_back({run.hxyz + 24 * p, fr[i].xyz, 24 * (size_t)fr[i].n});
        }
    }
    A.hd = (FrameDev *)h;
    h += r256(sizeof(FrameDev) * fr.size());
    A.ha = (int32_t *)h;
    for (size_t i = 0; i < fr.size(); ++i) {
        A.hd[i] = A.devs[i];
        A.ha[i] = A.slots[i];
    }
    if (copy) parallel_copy(jobs);
    return TBR_OK;
}

// Frame records and slot list up, scattered by one kernel.
static tbr_status upload_records(Engine &E, const StagedAdmission &A) {
    const size_t n = A.slots.size();
    TBR_CUDA(cudaMemcpyAsync(E.d_admit, A.hd, sizeof(FrameDev) * n, cudaMemcpyHostToDevice, E.stream));
    TBR_CUDA(cudaMemcpyAsync(E.d_active, A.ha, 4 * n, cudaMemcpyHostToDevice, E.stream));
    k_admit_frames<<<(int)n, 128, 0, E.stream>>>(E.P.frames, E.d_admit, E.d_active, (int)n);
    TBR_CUDA(cudaGetLastError());
    E.P.n_active = (int32_t)n;
    return TBR_OK;
}

// Device side of an admission whose host copies are done: one copy per run and array.
static tbr_status upload_staged(Engine &E, const StagedAdmission &A) {
    if (A.slots.empty()) return TBR_OK;
    for (auto &r : A.runs) {
        const size_t pts = (size_t)(r.b1 - r.b0) * kSub;
        const size_t p0 = (size_t)r.b0 * kSub;
        TBR_CUDA(cudaMemcpyAsync((void *)(E.P.uv64 + 2 * p0), r.huv, 16 * pts, cudaMemcpyHostToDevice, E.stream));
        TBR_CUDA(cudaMemcpyAsync((void *)(E.P.X64 + 3 * p0), r.hxyz, 24 * pts, cudaMemcpyHostToDevice, E.stream));
    }
    return upload_records(E, A);
}

// Host copies and uploads in groups of consecutive frames of a run, so that
// the link moves one group while the host threads copy the next: copy threads
// take 1 MiB pieces in group order, and this thread issues a group's upload as
// soon as its last piece is in.
// Large frames whose arrays are already page-locked go up directly, without a
// host copy (below ~512 KiB a copy into staging and a shared upload cost less
// than an upload call of their own).
constexpr size_t kDirectUploadBytes = 512u << 10;
static bool page_locked(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}
static bool direct_upload(const StagedAdmission &A, size_t i) {
    return A.jobs[2 * i].bytes + A.jobs[2 * i + 1].bytes >= kDirectUploadBytes && page_locked(A.jobs[2 * i].src) &&
           page_locked(A.jobs[2 * i + 1].src);
}

static tbr_status copy_and_upload_overlapped(Engine &E, const StagedAdmission &A) {
    constexpr size_t kGroupBytes = 8u << 20, kPiece = 1u << 20;
    struct Group {
        size_t run, i, j;  // frames i .. j-1 of run
    };
    std::vector<char> direct(A.devs.size(), 0);
    for (size_t i = 0; i < A.devs.size(); ++i) {
        direct[i] = direct_upload(A, i);
        if (direct[i]) {
            const size_t q0 = (size_t)A.devs[i].blk_off * kSub;
            TBR_CUDA(cudaMemcpyAsync((void *)(E.P.uv64 + 2 * q0), A.jobs[2 * i].src, A.jobs[2 * i].bytes,
                                     cudaMemcpyHostToDevice, E.stream));
            TBR_CUDA(cudaMemcpyAsync((void *)(E.P.X64 + 3 * q0), A.jobs[2 * i + 1].src, A.jobs[2 * i + 1].bytes,
                                     cudaMemcpyHostToDevice, E.stream));
        }
    }
    std::vector<Group> groups;
    size_t total = 0;
    for (size_t r = 0; r < A.runs.size(); ++r)
        for (size_t i = A.span[r].first; i <= A.span[r].second;) {
            if (direct[i]) {
                ++i;
                continue;
            }
            size_t j = i, bytes = 0;
            while (j <= A.span[r].second && !direct[j] && (j == i || bytes < kGroupBytes)) {
                bytes += A.jobs[2 * j].bytes + A.jobs[2 * j + 1].bytes;
                ++j;
            }
            groups.push_back({r, i, j});
            total += bytes;
            i = j;
        }
    auto upload = [&](const Group &g) -> tbr_status {
        const auto &run = A.runs[g.run];
        // points [p0, p1) of the run: the group's frames with their padding
        const size_t p0 = (size_t)(A.devs[g.i].blk_off - run.b0) * kSub;
        const size_t p1 = (size_t)(A.devs[g.j - 1].blk_off + A.devs[g.j - 1].n_blocks - run.b0) * kSub;
        const size_t q0 = (size_t)run.b0 * kSub + p0;
        TBR_CUDA(cudaMemcpyAsync((void *)(E.P.uv64 + 2 * q0), run.huv + 16 * p0, 16 * (p1 - p0),
                                 cudaMemcpyHostToDevice, E.stream));
        TBR_CUDA(cudaMemcpyAsync((void *)(E.P.X64 + 3 * q0), run.hxyz + 24 * p0, 24 * (p1 - p0),
                                 cudaMemcpyHostToDevice, E.stream));
        return TBR_OK;
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int T = (int)std::min<size_t>(std::min(8u, hw), total / (4 * kPiece));
    if (T <= 1) {
        for (auto &g : groups) {
            for (size_t k = 2 * g.i; k < 2 * g.j; ++k) std::memcpy(A.jobs[k].dst, A.jobs[k].src, A.jobs[k].bytes);
            tbr_status st = upload(g);
            if (st) return st;
        }
        return upload_records(E, A);
    }
    struct Piece {
        CopyJob job;
        size_t group;
    };
    std::vector<Piece> pieces;
    std::unique_ptr<std::atomic<int>[]> left(new std::atomic<int>[groups.size()]);
    for (size_t g = 0; g < groups.size(); ++g) {
        int cnt = 0;
        for (size_t k = 2 * groups[g].i; k < 2 * groups[g].j; ++k)
            for (size_t o = 0; o < A.jobs[k].bytes; o += kPiece, ++cnt)
                pieces.push_back({{(char *)A.jobs[k].dst + o, (const char *)A.jobs[k].src + o,
                                   std::min(kPiece, A.jobs[k].bytes - o)},
                                  g});
        left[g].store(cnt, std::memory_order_relaxed);
    }
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t k; (k = next.fetch_add(1)) < pieces.size();) {
            std::memcpy(pieces[k].job.dst, pieces[k].job.src, pieces[k].job.bytes);
            left[pieces[k].group].fetch_sub(1, std::memory_order_release);
        }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) th.emplace_back(work);
    tbr_status st = TBR_OK;
    for (size_t g = 0; g < groups.size(); ++g) {
        while (left[g].load(std::memory_order_acquire) > 0) std::this_thread::yield();
        if (st == TBR_OK) st = upload(groups[g]);
    }
    for (auto &x : th) x.join();
    if (st) return st;
    return upload_records(E, A);
}

// ------------------------------------------------------ ingestion tables --
// Tiles of one (source, pool destination) row, at most `tile` bytes each.
static void add_row_tiles(std::vector<IngestTile> &v, const void *src, const void *dst, size_t bytes, size_t tile) {
    for (size_t o = 0; o < bytes; o += tile)
        v.push_back({(const char *)src + o, (char *)dst + o, (int64_t)std::min(tile, bytes - o)});
}
// Frame k's two rows: uv into the pool's uv64, xyz into X64.
static void add_frame_tiles(std::vector<IngestTile> &v, const Engine &E, const FrameDev &d, int64_t n,
                            const void *src_uv, const void *src_xyz, size_t tile) {
    const size_t q0 = (size_t)d.blk_off * kSub;
    add_row_tiles(v, src_uv, E.P.uv64 + 2 * q0, 16 * (size_t)n, tile);
    add_row_tiles(v, src_xyz, E.P.X64 + 3 * q0, 24 * (size_t)n, tile);
}
// Tile size that keeps every table of one call within d_ingest.
static size_t ingest_tile_bytes(const std::vector<FrameHost> &fr) {
    size_t tile = kIngestTileBytes;
    for (;;) {
        size_t cnt = 0;
        for (auto &f : fr) cnt += (16 * (size_t)f.n + tile - 1) / tile + (24 * (size_t)f.n + tile - 1) / tile;
        if (cnt <= (size_t)kIngestTileCap) return tile;
        tile *= 2;
    }
}
// Writes a table (count header + tiles) at byte `off` of the pinned mirror
// `h` and enqueues its upload to the same offset of d_ingest; returns the
// device address of the table and advances `off`.
static const int64_t *put_table(Engine &E, char *h, size_t &off, const std::vector<IngestTile> &t,
                                 char *d_tables, cudaStream_t st) {
    if (off + 16 + sizeof(IngestTile) * t.size() > Engine::kIngestTableBytes) return nullptr;
    int64_t *hdr = (int64_t *)(h + off);
    hdr[0] = (int64_t)t.size();
    hdr[1] = 0;
    if (!t.empty()) std::memcpy(hdr + 2, t.data(), sizeof(IngestTile) * t.size());
    const size_t bytes = 16 + sizeof(IngestTile) * t.size();
    const int64_t *d = (const int64_t *)(d_tables + off);
    if (cudaMemcpyAsync((void *)d, hdr, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) return nullptr;
    off += (bytes + 15) & ~size_t(15);
    return d;
}
// Device address of page-locked host memory (nullptr for pageable memory).
static const void *mapped_address(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return at.type == cudaMemoryTypeHost ? at.devicePointer : nullptr;
}

// Host-buffer admission by zero-copy ingestion: every frame's arrays are read
// by k_ingest over the link, from the caller's memory when it is page-locked,
// else from a staging copy made by the host threads. Frames are ingested in
// groups of about kIngestGroupBytes of staged data, so the link moves one
// group while the host threads copy the next; page-locked frames cost no host
// work at all, and no per-frame copy call is issued.
//
// With `launch`, the call also starts the run and overlaps it with the
// ingestion: the frames are split, in order, and only the first part (about
// kStaggerFirstShare of the bytes) is ingested and prepared before the loop
// graph starts; the rest is admitted kPending and ingested and prepared by the
// graph itself beside the first engine step, and starts RANSAC in the second
// (a frame's samples and results do not depend on the step it starts in).
// The first part is ingested on stream_in, so that it overlaps whatever the
// context stream still runs (a batch submitted before); the context stream
// waits for it before the preparation. E.ev0 then marks the start of the
// first part's preparation. Without `stagger` (a submission queued behind
// another batch, whose run hides the ingestion) every frame is in the first
// part and the plain loop graph runs.
//
// `slots`, `max_n` and `devs` are set as soon as the frames hold slots (the
// caller releases them whatever happens next).
constexpr size_t kZeroCopyMinBytes = 4u << 20;
constexpr size_t kIngestGroupBytes = 8u << 20;
constexpr size_t kStaggerMinBytes = 16u << 20;
constexpr double kStaggerFirstShare = 0.35;

static tbr_status admit_host_frames(Engine &E, const std::vector<FrameHost> &fr, const RunOptions &o,
                                    std::vector<int> &slots, int64_t &max_n, std::vector<FrameDev> &devs,
                                    bool launch, bool stagger = true) {
    constexpr size_t kPiece = 1u << 20;
    const size_t n = fr.size();
    const size_t tab_off = stage_bytes(fr);
    tbr_status st = E.ensure_stage(tab_off + Engine::kIngestTableBytes);
    if (st) return st;
    StagedAdmission A;
    st = stage_frames(E, fr, o, (char *)E.h_stage, A, false, true);
    if (st) return st;
    slots = A.slots;
    max_n = A.max_n;
    devs = A.devs;
    if (!E.d_stage_alias) return fail(TBR_ERR_CUDA, "staging buffer has no device address");
    // Sources as the device sees them.
    std::vector<const void *> su(n), sx(n);
    std::vector<char> staged(n, 0);
    std::vector<size_t> fb(n);
    size_t total = 0;
    for (size_t k = 0; k < n; ++k) {
        total += (fb[k] = A.jobs[2 * k].bytes + A.jobs[2 * k + 1].bytes);
        su[k] = mapped_address(fr[k].uv);
        sx[k] = su[k] ? mapped_address(fr[k].xyz) : nullptr;
        if (!su[k] || !sx[k]) {
            staged[k] = 1;
            su[k] = (const char *)E.d_stage_alias + ((const char *)A.jobs[2 * k].dst - (const char *)E.h_stage);
            sx[k] = (const char *)E.d_stage_alias + ((const char *)A.jobs[2 * k + 1].dst - (const char *)E.h_stage);
        }
    }
    size_t n_first = n;
    Engine::Stagger sg;
    if (launch && stagger) {
        size_t acc = 0;
        const size_t first = (size_t)(kStaggerFirstShare * (double)total);
        n_first = 0;
        while (n_first < n && (n_first == 0 || acc < first)) acc += fb[n_first++];
        if (n_first == n) n_first = n - 1;  // at least one late frame
        sg.n_first = (int)n_first;
        for (size_t k = n_first; k < n; ++k) {
            A.hd[k].status = kPending;
            sg.max_n_rest = std::max(sg.max_n_rest, fr[k].n);
        }
    }
    // Ingestion groups of the first part: [gb[g], gb[g + 1]); at most about
    // 60 tables, so that their headers fit d_ingest.
    size_t staged_total = 0;
    for (size_t k = 0; k < n_first; ++k) staged_total += staged[k] ? fb[k] : 0;
    const size_t group_bytes = std::max(kIngestGroupBytes, staged_total / 60 + 1);
    std::vector<size_t> gb{0};
    for (size_t k = 0, acc = 0; k < n_first; ++k) {
        acc += staged[k] ? fb[k] : 0;
        if (acc >= group_bytes || k + 1 == n_first) {
            gb.push_back(k + 1);
            acc = 0;
        }
    }
    const size_t G = gb.size() - 1;  // the late frames are group G
    struct Piece {
        CopyJob job;
        size_t group;
    };
    std::vector<Piece> pieces;
    std::unique_ptr<std::atomic<int>[]> left(new std::atomic<int>[G + 1]);
    for (size_t g = 0; g <= G; ++g) {
        const size_t k0 = g < G ? gb[g] : n_first, k1 = g < G ? gb[g + 1] : n;
        int cnt = 0;
        for (size_t k = k0; k < k1; ++k)
            if (staged[k])
                for (size_t jb = 2 * k; jb < 2 * k + 2; ++jb)
                    for (size_t off = 0; off < A.jobs[jb].bytes; off += kPiece, ++cnt)
                        pieces.push_back({{(char *)A.jobs[jb].dst + off, (const char *)A.jobs[jb].src + off,
                                           std::min(kPiece, A.jobs[jb].bytes - off)},
                                          g});
        left[g].store(cnt, std::memory_order_relaxed);
    }
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t k; (k = next.fetch_add(1)) < pieces.size();) {
            std::memcpy(pieces[k].job.dst, pieces[k].job.src, pieces[k].job.bytes);
            left[pieces[k].group].fetch_sub(1, std::memory_order_release);
        }
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> th;
    const size_t staged_bytes = pieces.size() * kPiece;
    if (staged_bytes >= 4 * kPiece)
        for (unsigned t = 0; t < std::min(8u, hw); ++t) th.emplace_back(work);
    else
        work();  // little to copy: this thread does it
    auto wait_group = [&](size_t g) {
        while (left[g].load(std::memory_order_acquire) > 0) std::this_thread::yield();
    };
    const size_t tile = ingest_tile_bytes(fr);
    // With `launch` the first part is ingested on stream_in, beside the work
    // still queued on the context stream (the new frames' blocks and their
    // tables are this call's alone).
    cudaStream_t in = launch ? E.stream_in : E.stream;
    auto enqueue = [&]() -> tbr_status {
        tbr_status s2 = upload_records(E, A);
        if (s2) return s2;
        char *h = (char *)E.h_stage + tab_off;
        // The late frames' table sits at offset 0, where the graph reads it;
        // the first part's tables follow it.
        std::vector<IngestTile> late;
        if (launch)
            for (size_t k = n_first; k < n; ++k) add_frame_tiles(late, E, A.devs[k], fr[k].n, su[k], sx[k], tile);
        size_t off = launch ? ((16 + sizeof(IngestTile) * late.size() + 15) & ~size_t(15)) : 0;
        std::vector<IngestTile> t;
        for (size_t g = 0; g < G; ++g) {
            t.clear();
            for (size_t k = gb[g]; k < gb[g + 1]; ++k) add_frame_tiles(t, E, A.devs[k], fr[k].n, su[k], sx[k], tile);
            wait_group(g);
            const int64_t *d = put_table(E, h, off, t, launch ? E.d_ingest_first : E.d_ingest, in);
            if (!d) return fail(TBR_ERR_CUDA, "ingestion table upload failed");
            k_ingest<<<stagger ? Engine::kIngestGridHost : Engine::kIngestGridBeside, 256, 0, in>>>(d);
            TBR_CUDA(cudaGetLastError());
        }
        if (!launch) return TBR_OK;
        TBR_CUDA(cudaEventRecord(E.ev_in, in));
        TBR_CUDA(cudaStreamWaitEvent(E.stream, E.ev_in, 0));
        if (stagger) {
            size_t off0 = 0;
            wait_group(G);  // the graph reads the late frames' staging copies
            if (!put_table(E, h, off0, late, E.d_ingest, E.stream))
                return fail(TBR_ERR_CUDA, "ingestion table upload failed");
        }
        TBR_CUDA(cudaEventRecord(E.ev0, E.stream));
        Pools Qf = E.P;
        Qf.n_active = (int32_t)n_first;
        int64_t max_first = 0;
        for (size_t k = 0; k < n_first; ++k) max_first = std::max(max_first, fr[k].n);
        E.launch_prep(Qf, (int)n_first, max_first, E.stream);
        E.pp = o.pp;
        return E.launch_graph((int)n, o.hr, stagger ? &sg : nullptr);
    };
    st = enqueue();
    for (auto &x : th) x.join();
    return st;
}

// Both halves through the context's own staging buffer. With device_points the
// frames' point arrays are device memory of this GPU: they are copied into the
// pool by one kernel, with no host staging. Multi-frame host batches of some
// size are ingested zero-copy (admit_host_frames); a small admission uploads
// its staging runs with copy calls.
static tbr_status admit_frames(Engine &E, const std::vector<FrameHost> &fr, const RunOptions &o,
                               std::vector<int> &slots, int64_t &max_n, std::vector<FrameDev> *host_devs = nullptr,
                               bool device_points = false) {
    size_t in_bytes = 0;
    for (auto &f : fr) in_bytes += 40 * (size_t)f.n;
    if (!device_points && fr.size() >= 2 && in_bytes >= kZeroCopyMinBytes) {
        std::vector<FrameDev> d;
        tbr_status st = admit_host_frames(E, fr, o, slots, max_n, d, false);
        if (host_devs) *host_devs = d;
        return st;
    }
    auto r256 = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t rec = r256(sizeof(FrameDev) * fr.size()) + r256(4 * fr.size());
    tbr_status st = E.ensure_stage(device_points ? rec + Engine::kIngestTableBytes : stage_bytes(fr));
    if (st) return st;
    StagedAdmission A;
    st = stage_frames(E, fr, o, (char *)E.h_stage, A, false, !device_points);
    if (st) return st;
    // The caller releases these, whatever happens next.
    slots = A.slots;
    max_n = A.max_n;
    if (host_devs) *host_devs = A.devs;
    if (device_points) {
        std::vector<IngestTile> t;
        const size_t tile = ingest_tile_bytes(fr);
        for (size_t i = 0; i < fr.size(); ++i) add_frame_tiles(t, E, A.devs[i], fr[i].n, fr[i].uv, fr[i].xyz, tile);
        size_t off = 0;
        const int64_t *d = put_table(E, (char *)E.h_stage + rec, off, t, E.d_ingest, E.stream);
        if (!d) return fail(TBR_ERR_CUDA, "ingestion table upload failed");
        k_ingest<<<E.num_sms * 2, 256, 0, E.stream>>>(d);
        TBR_CUDA(cudaGetLastError());
        st = upload_records(E, A);
    } else {
        st = copy_and_upload_overlapped(E, A);
    }
    return st;
}

// Results of `slots` into `out` (host), through one packed download.
static tbr_status fetch_results(Engine &E, const std::vector<int> &slots, FrameResult *out) {
    const size_t n = slots.size();
    if (n == 0) return TBR_OK;
    tbr_status st = E.ensure_stage(sizeof(FrameResult) * n + 4 * n + 512);
    if (st) return st;
    FrameResult *hres = (FrameResult *)E.h_stage;
    int32_t *hs = (int32_t *)((char *)E.h_stage + ((sizeof(FrameResult) * n + 255) & ~size_t(255)));
    for (size_t i = 0; i < n; ++i) hs[i] = slots[i];
    int32_t *ds = E.d_res_slots;
    TBR_CUDA(cudaMemcpyAsync(ds, hs, 4 * n, cudaMemcpyHostToDevice, E.stream));
    k_gather_results<<<(int)std::min<size_t>(1024, (n * (sizeof(FrameResult) / 8) + 255) / 256), 256, 0, E.stream>>>(
        E.P.results, ds, (int)n, E.d_res_stage);
    TBR_CUDA(cudaGetLastError());
    TBR_CUDA(cudaMemcpyAsync(hres, E.d_res_stage, sizeof(FrameResult) * n, cudaMemcpyDeviceToHost, E.stream));
    TBR_CUDA(cudaStreamSynchronize(E.stream));
    std::memcpy(out, hres, sizeof(FrameResult) * n);
    return TBR_OK;
}

static void fill_stats(const FrameResult &r, int64_t n, tbr_stats *st, float ms) {
    if (!st) return;
    st->samples = r.samples;
    st->rounds = r.rounds;
    st->hypotheses = r.hypotheses;
    st->ransac_inliers = r.ransac_inliers;
    st->num_inliers = r.num_inliers;
    st->inlier_ratio = n > 0 ? (double)r.num_inliers / (double)n : 0.0;
    st->model_score = r.model_score;
    st->best_sample = r.best_sample;
    st->best_solution = r.best_sol;
    st->steps = r.steps;
    st->candidates_rescored = r.rescored;
    st->candidate_overflow = r.overflow;
    st->lm_iterations = r.lm_iters;
    st->lm_invalid_steps = r.lm_invalid;
    st->lm_initial_cost = r.lm_cost0;
    st->lm_cost = r.lm_cost;
    st->gpu_ms = ms;
}

}  // namespace tbr

using namespace tbr;

struct tbr_context {
    Engine E;
    std::vector<tbr_ticket *> tickets;  // submitted, not yet collected
};

// A submitted batch: its frames' slots and workspace blocks (held until
// collect), the call-buffer set its queued downloads land in, and, once
// retired (its device work waited for), its results.
struct tbr_ticket {
    tbr_context *ctx = nullptr;
    int set = -1;  // call-buffer set of its queued work; -1 once retired
    std::vector<int> slots;
    std::vector<FrameDev> devs;
    std::vector<int64_t> ns;
    std::vector<FrameResult> res;
    tbr_status st = TBR_OK;
    std::string msg;
    float ms = 0.f;
};

struct tbr_batch;
static void destroy_context_batches(tbr_context *ctx);

// The device run's verdict from its downloaded counters.
static tbr_status run_status(const unsigned long long *counters) {
    if (counters[kCError] & kErrTimeout) return fail(TBR_ERR_TIMEOUT, "bounded device wait expired");
    if (counters[kCError] & kErrOverflow) return fail(TBR_ERR_INTERNAL, "step limit or capacity exceeded");
    return TBR_OK;
}

static void release_frames(Engine &E, const std::vector<int> &slots, const std::vector<FrameDev> &devs) {
    for (size_t i = 0; i < slots.size(); ++i) {
        E.blocks.release(devs[i].blk_off, devs[i].n_blocks);
        E.free_slots.push_back(slots[i]);
    }
}

static std::mutex g_tickets_mu;
static std::unordered_map<tbr_ticket *, tbr_context *> g_tickets;

// Waits for a submitted batch's device work and moves its results out of the
// call buffers, which are then free for the next submission. Context lock held.
static void retire_ticket(tbr_ticket *t) {
    if (t->set < 0) return;
    Engine &E = t->ctx->E;
    E.bind_set(t->set);
    const cudaError_t e = cudaEventSynchronize(E.ev_done);
    if (e != cudaSuccess) {
        t->st = TBR_ERR_CUDA;
        t->msg = std::string("cudaEventSynchronize: ") + cudaGetErrorString(e);
    } else if ((t->st = run_status(E.h_counters)) != TBR_OK) {
        t->msg = g_last_error;
    } else {
        t->res.assign(E.h_results, E.h_results + t->slots.size());
        cudaEventElapsedTime(&t->ms, E.ev0, E.ev1);
    }
    E.owner[t->set] = nullptr;
    t->set = -1;
}
// Every entry point other than submit and collect starts here (context lock
// held): the shared call buffers are free afterwards.
static void retire_tickets(tbr_context *ctx) {
    for (tbr_ticket *t : ctx->tickets) retire_ticket(t);
}
static void destroy_context_tickets(tbr_context *ctx) {
    std::lock_guard<std::mutex> lk(ctx->E.mu);
    cudaStreamSynchronize(ctx->E.stream);
    for (tbr_ticket *t : ctx->tickets) {
        {
            std::lock_guard<std::mutex> g(g_tickets_mu);
            g_tickets.erase(t);
        }
        delete t;
    }
    ctx->tickets.clear();
    ctx->E.owner[0] = ctx->E.owner[1] = nullptr;
}

// =================================================================== C ABI ==
extern "C" {

int tbr_abi_version(void) { return TBR_ABI_VERSION; }
const char *tbr_last_error(void) { return g_last_error.c_str(); }

void tbr_default_ransac_options(tbr_ransac_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->max_iterations = 100000;
    o->min_iterations = 1000;
    o->dyn_num_trials_mult = 3.0;
    o->success_prob = 0.9999;
    o->max_reproj_error = 12.0;
    o->max_epipolar_error = 1.0;
    o->seed = 0;
    o->max_prosac_iterations = 100000;
}

void tbr_default_bundle_options(tbr_bundle_options *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->max_iterations = 100;
    o->loss_type = 3;
    o->loss_scale = 1.0;
    o->gradient_tol = 1e-10;
    o->step_tol = 1e-8;
    o->initial_lambda = 1e-3;
    o->min_lambda = 1e-10;
    o->max_lambda = 1e10;
}

tbr_status tbr_context_create(int device, uint64_t workspace_bytes, tbr_context **out) {
    if (!out) return fail(TBR_ERR_INVALID_ARG, "out is NULL");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(TBR_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev) return fail(TBR_ERR_INVALID_ARG, "bad device ordinal");
    auto *c = new tbr_context();
    tbr_status s = c->E.init(device, workspace_bytes);
    if (s != TBR_OK) {
        delete c;
        return s;
    }
    *out = c;
    return TBR_OK;
}

void tbr_context_destroy(tbr_context *ctx) {
    if (!ctx) return;
    destroy_context_batches(ctx);
    destroy_context_tickets(ctx);
    delete ctx;
}

// Queues a whole run of the frames on the context's stream and returns: the
// admission (for a large host batch, ingestion overlapped with the first
// step, or -- `behind` another queued batch -- with that batch's run), the
// loop graph, then the results' gather and their download, with the
// counters, into the bound call buffers (ev0 / ev1 bracket the device run).
// `slots` and `devs` are set as soon as the frames hold them, whatever happens
// next (the caller releases them).
static tbr_status enqueue_frames(Engine &E, const std::vector<FrameHost> &fr, const RunOptions &o,
                                 std::vector<int> &slots, std::vector<FrameDev> &devs, bool device_points,
                                 bool behind = false) {
    int64_t max_n = 0;
    TBR_CUDA(cudaSetDevice(E.device));
    TBR_CUDA(cudaMemsetAsync(E.P.counters, 0, 8 * kCNum, E.stream));
    size_t in_bytes = 0;
    for (auto &f : fr) in_bytes += 40 * (size_t)f.n;
    tbr_status st;
    if (!device_points && fr.size() >= 2 && in_bytes >= kStaggerMinBytes) {
        st = admit_host_frames(E, fr, o, slots, max_n, devs, true, !behind);
    } else {
        st = admit_frames(E, fr, o, slots, max_n, &devs, device_points);
        if (st == TBR_OK) {
            TBR_CUDA(cudaEventRecord(E.ev0, E.stream));
            E.launch_prep((int)slots.size(), max_n);
            E.pp = o.pp;
            st = E.launch_graph((int)slots.size(), o.hr);
        }
    }
    if (st) return st;
    TBR_CUDA(cudaEventRecord(E.ev1, E.stream));
    // Everything the caller gets back in one round trip: the results in the
    // order of the active list (= slots) and the counters.
    const int n = (int)slots.size();
    k_gather_results<<<(int)std::min<size_t>(1024, (n * (sizeof(FrameResult) / 8) + 255) / 256), 256, 0,
                       E.stream>>>(E.P.results, E.d_active, n, E.d_res_stage);
    TBR_CUDA(cudaGetLastError());
    TBR_CUDA(cudaMemcpyAsync(E.h_results, E.d_res_stage, sizeof(FrameResult) * n, cudaMemcpyDeviceToHost,
                             E.stream));
    TBR_CUDA(cudaMemcpyAsync(E.h_counters, E.P.counters, 8 * kCNum, cudaMemcpyDeviceToHost, E.stream));
    return TBR_OK;
}

static tbr_status estimate_frames(tbr_context *ctx, const std::vector<FrameHost> &fr, const RunOptions &o,
                                  std::vector<FrameResult> &res, std::vector<uint8_t *> masks,
                                  float *ms_out, int *steps_out, bool device_points = false) {
    Engine &E = ctx->E;
    std::vector<int> slots;
    std::vector<FrameDev> devs;
    tbr_status st = enqueue_frames(E, fr, o, slots, devs, device_points);
    if (st == TBR_OK) {
        for (size_t i = 0; i < slots.size(); ++i)
            if (i < masks.size() && masks[i])
                TBR_CUDA(cudaMemcpyAsync(masks[i], E.P.mask + devs[i].blk_off * kSub, fr[i].n,
                                         cudaMemcpyDeviceToHost, E.stream));
        TBR_CUDA(cudaStreamSynchronize(E.stream));
        st = run_status(E.h_counters);
        if (st == TBR_OK) {
            res.assign(E.h_results, E.h_results + slots.size());
            if (steps_out) *steps_out = (int)E.h_counters[kCSteps];
            float ms = 0.f;
            cudaEventElapsedTime(&ms, E.ev0, E.ev1);
            if (ms_out) *ms_out = ms;
        }
    }
    cudaStreamSynchronize(E.stream);
    cudaStreamSynchronize(E.stream_in);  // an admission that failed may have left ingestion queued there
    release_frames(E, slots, devs);
    return st;
}

tbr_status tbr_estimate_absolute_pose(tbr_context *ctx, const double *points2D, const double *points3D,
                                      int64_t n, const double K[4], int32_t width, int32_t height,
                                      const tbr_ransac_options *ransac_opt,
                                      const tbr_bundle_options *bundle_opt, const tbr_ext_options *ext,
                                      double q[4], double t[3], uint8_t *inliers, tbr_stats *stats) {
    (void)width;
    (void)height;
    if (!ctx || !points2D || !points3D || !K || !q || !t) return fail(TBR_ERR_INVALID_ARG, "NULL argument");
    if (n < 3) return fail(TBR_ERR_INVALID_ARG, "need at least 3 correspondences");
    if (!(K[0] > 0) || !(K[1] > 0)) return fail(TBR_ERR_INVALID_ARG, "focal lengths must be positive");
    tbr_ransac_options ro;
    tbr_default_ransac_options(&ro);
    if (ransac_opt) ro = *ransac_opt;
    if (ro.max_iterations < 1) return fail(TBR_ERR_INVALID_ARG, "max_iterations (samples per round) must be >= 1");
    if (!(ro.max_reproj_error > 0)) return fail(TBR_ERR_INVALID_ARG, "max_reproj_error must be > 0");
    RunOptions o = make_run_options(&ro, bundle_opt, ext);
    FrameHost fh{points2D, points3D, n, {K[0], K[1], K[2], K[3]}, ro.seed, ro.max_reproj_error, nullptr, 0};
    if (ext && ext->seed) fh.seed = ext->seed;
    if (ext && ext->replay_idx) {
        if (ext->replay_count < 1) return fail(TBR_ERR_INVALID_ARG, "empty replay buffer");
        for (int64_t i = 0; i < 3 * ext->replay_count; ++i)
            if (ext->replay_idx[i] < 0 || ext->replay_idx[i] >= n)
                return fail(TBR_ERR_INVALID_ARG, "replayed index out of range");
        if (o.force_samples > 0) {
            if (o.force_samples > ext->replay_count)
                return fail(TBR_ERR_INVALID_ARG, "replay buffer shorter than force_samples");
        } else {
            // Rounds always draw B samples; a replayed run stops at the last full round.
            if (ext->replay_count < o.B) return fail(TBR_ERR_INVALID_ARG, "replay buffer shorter than one round");
            o.max_total = std::min<int64_t>(o.max_total, (ext->replay_count / o.B) * o.B);
        }
        fh.replay = ext->replay_idx;
        fh.replay_count = ext->replay_count;
    }
    std::lock_guard<std::mutex> lk(ctx->E.mu);
    retire_tickets(ctx);
    std::vector<FrameResult> res;
    float ms = 0.f;
    int steps = 0;
    tbr_status st = estimate_frames(ctx, {fh}, o, res, {inliers}, &ms, &steps);
    if (st) return st;
    for (int k = 0; k < 4; ++k) q[k] = res[0].q[k];
    for (int k = 0; k < 3; ++k) t[k] = res[0].t[k];
    fill_stats(res[0], n, stats, ms);
    return TBR_OK;
}

}  // extern "C"

// Frames beyond what the context holds at once run in consecutive groups of
// at most its frame capacity; each frame's result does not depend on the
// grouping.
static tbr_status estimate_frames_chunked(tbr_context *ctx, const std::vector<FrameHost> &fr, const RunOptions &o,
                                          std::vector<FrameResult> &res, const std::vector<uint8_t *> &masks,
                                          std::vector<float> &ms, bool device_points) {
    const size_t cap = (size_t)std::max(1, ctx->E.max_frames);
    res.clear();
    ms.assign(fr.size(), 0.f);
    for (size_t i0 = 0; i0 < fr.size(); i0 += cap) {
        const size_t i1 = std::min(fr.size(), i0 + cap);
        std::vector<FrameHost> sub(fr.begin() + i0, fr.begin() + i1);
        std::vector<uint8_t *> sm(masks.begin() + i0, masks.begin() + i1);
        std::vector<FrameResult> r;
        float t = 0.f;
        int steps = 0;
        tbr_status st = estimate_frames(ctx, sub, o, r, sm, &t, &steps, device_points);
        if (st) return st;
        res.insert(res.end(), r.begin(), r.end());
        for (size_t i = i0; i < i1; ++i) ms[i] = t;
    }
    return TBR_OK;
}

// Argument checks shared by the batched entry points, the same as the plain
// call's: at least one sample per round, a positive threshold, and per frame
// three correspondences, both arrays and positive focal lengths.
static tbr_status check_ransac(const tbr_ransac_options &ro) {
    if (ro.max_iterations < 1) return fail(TBR_ERR_INVALID_ARG, "max_iterations (samples per round) must be >= 1");
    if (!(ro.max_reproj_error > 0)) return fail(TBR_ERR_INVALID_ARG, "max_reproj_error must be > 0");
    return TBR_OK;
}
static tbr_status check_frame(const tbr_frame_desc &d) {
    if (d.n < 3 || !d.points2D || !d.points3D) return fail(TBR_ERR_INVALID_ARG, "bad frame");
    if (!(d.K[0] > 0) || !(d.K[1] > 0)) return fail(TBR_ERR_INVALID_ARG, "bad camera");
    return TBR_OK;
}
static FrameHost frame_host(const tbr_frame_desc &d, const tbr_ransac_options &ro) {
    return {d.points2D, d.points3D, d.n, {d.K[0], d.K[1], d.K[2], d.K[3]}, d.seed,
            d.max_reproj_error > 0 ? d.max_reproj_error : ro.max_reproj_error, nullptr, 0};
}
// The device-input calls' frames: the plain call's checks, and both arrays
// device memory of the context's GPU.
static tbr_status device_frames(Engine &E, const tbr_frame_desc *frames, int32_t n, const tbr_ransac_options &ro,
                                std::vector<FrameHost> &fr) {
    for (int i = 0; i < n; ++i) {
        const tbr_frame_desc &d = frames[i];
        if (tbr_status c = check_frame(d)) return c;
        for (const void *p : {(const void *)d.points2D, (const void *)d.points3D}) {
            cudaPointerAttributes a;
            if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
                cudaGetLastError();
                return fail(TBR_ERR_INVALID_ARG, "frame points are not device memory");
            }
            if ((a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) || a.device != E.device)
                return fail(TBR_ERR_INVALID_ARG, "frame points are not device memory of the context's GPU");
        }
        fr.push_back(frame_host(d, ro));
    }
    return TBR_OK;
}

extern "C" {

tbr_status tbr_estimate_batch(tbr_context *ctx, const tbr_frame_desc *frames, int32_t n_frames,
                              const tbr_ransac_options *ransac_opt, const tbr_ext_options *ext,
                              tbr_frame_result *results, uint8_t *const *inliers) {
    if (!ctx || !frames || n_frames < 1 || !results) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    tbr_ransac_options ro;
    tbr_default_ransac_options(&ro);
    if (ransac_opt) ro = *ransac_opt;
    if (tbr_status c = check_ransac(ro)) return c;
    RunOptions o = make_run_options(&ro, nullptr, ext);
    std::vector<FrameHost> fr;
    for (int i = 0; i < n_frames; ++i) {
        if (tbr_status c = check_frame(frames[i])) return c;
        fr.push_back(frame_host(frames[i], ro));
    }
    std::lock_guard<std::mutex> lk(ctx->E.mu);
    retire_tickets(ctx);
    std::vector<FrameResult> res;
    std::vector<uint8_t *> masks(n_frames, nullptr);
    if (inliers)
        for (int i = 0; i < n_frames; ++i) masks[i] = inliers[i];
    std::vector<float> ms;
    tbr_status st = estimate_frames_chunked(ctx, fr, o, res, masks, ms, false);
    if (st) return st;
    for (int i = 0; i < n_frames; ++i) {
        for (int k = 0; k < 4; ++k) results[i].q[k] = res[i].q[k];
        for (int k = 0; k < 3; ++k) results[i].t[k] = res[i].t[k];
        results[i].status = TBR_OK;
        fill_stats(res[i], fr[i].n, &results[i].stats, ms[i]);
    }
    return TBR_OK;
}

tbr_status tbr_estimate_batch_device(tbr_context *ctx, const tbr_frame_desc *frames, int32_t n_frames,
                                     const tbr_ransac_options *ransac_opt, const tbr_ext_options *ext,
                                     void *stream, tbr_frame_result *results, uint8_t *const *inliers) {
    if (!ctx || !frames || n_frames < 1 || !results) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    tbr_ransac_options ro;
    tbr_default_ransac_options(&ro);
    if (ransac_opt) ro = *ransac_opt;
    if (tbr_status c = check_ransac(ro)) return c;
    RunOptions o = make_run_options(&ro, nullptr, ext);
    Engine &E = ctx->E;
    std::vector<FrameHost> fr;
    if (tbr_status c = device_frames(E, frames, n_frames, ro, fr)) return c;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(ctx);
    TBR_CUDA(cudaSetDevice(E.device));
    if (stream) {  // the producer's pending writes come first
        TBR_CUDA(cudaEventRecord(E.ev_ingest, (cudaStream_t)stream));
        TBR_CUDA(cudaStreamWaitEvent(E.stream, E.ev_ingest, 0));
    }
    std::vector<FrameResult> res;
    std::vector<uint8_t *> masks(n_frames, nullptr);
    if (inliers)
        for (int i = 0; i < n_frames; ++i) masks[i] = inliers[i];
    std::vector<float> ms;
    tbr_status st = estimate_frames_chunked(ctx, fr, o, res, masks, ms, true);
    if (st) return st;
    for (int i = 0; i < n_frames; ++i) {
        for (int k = 0; k < 4; ++k) results[i].q[k] = res[i].q[k];
        for (int k = 0; k < 3; ++k) results[i].t[k] = res[i].t[k];
        results[i].status = TBR_OK;
        fill_stats(res[i], fr[i].n, &results[i].stats, ms[i]);
    }
    return TBR_OK;
}

}  // extern "C"

// The locked half of both submit calls: queue the run on the next call-buffer
// set and hand out its ticket. With device_points the frames' arrays are
// device memory, copied after the work queued on `stream` (if any).
static tbr_status submit_frames(tbr_context *ctx, const std::vector<FrameHost> &fr, const RunOptions &o,
                                bool device_points, void *stream, tbr_ticket **ticket) {
    std::lock_guard<std::mutex> lk(ctx->E.mu);
    Engine &E = ctx->E;
    const int k = E.next_set;
    if (E.owner[k]) retire_ticket(E.owner[k]);  // the oldest submission's downloads use set k
    E.bind_set(k);
    if (device_points && stream) {  // the producer's pending writes come first
        TBR_CUDA(cudaSetDevice(E.device));
        TBR_CUDA(cudaEventRecord(E.ev_ingest, (cudaStream_t)stream));
        TBR_CUDA(cudaStreamWaitEvent(E.stream, E.ev_ingest, 0));
    }
    std::unique_ptr<tbr_ticket> t(new tbr_ticket);
    // Queued behind the other set's batch (not yet waited for): that run
    // hides this one's whole ingestion, so no staggered start.
    tbr_status st = enqueue_frames(E, fr, o, t->slots, t->devs, device_points, E.owner[k ^ 1] != nullptr);
    if (st == TBR_OK) {
        const cudaError_t e = cudaEventRecord(E.ev_done, E.stream);
        if (e != cudaSuccess) st = fail(TBR_ERR_CUDA, std::string("cudaEventRecord: ") + cudaGetErrorString(e));
    }
    if (st) {
        cudaStreamSynchronize(E.stream);
        cudaStreamSynchronize(E.stream_in);  // an admission that failed may have left ingestion queued there
        release_frames(E, t->slots, t->devs);
        return st;
    }
    t->ctx = ctx;
    t->set = k;
    for (auto &f : fr) t->ns.push_back(f.n);
    E.owner[k] = t.get();
    E.next_set = k ^ 1;
    ctx->tickets.push_back(t.get());
    {
        std::lock_guard<std::mutex> g(g_tickets_mu);
        g_tickets[t.get()] = ctx;
    }
    *ticket = t.release();
    return TBR_OK;
}

extern "C" {

tbr_status tbr_estimate_batch_submit(tbr_context *ctx, const tbr_frame_desc *frames, int32_t n_frames,
                                     const tbr_ransac_options *ransac_opt, const tbr_ext_options *ext,
                                     tbr_ticket **ticket) {
    if (!ctx || !frames || n_frames < 1 || !ticket) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    *ticket = nullptr;
    if (n_frames > kMaxActive) return fail(TBR_ERR_INVALID_ARG, "more than 1024 frames in one submission");
    tbr_ransac_options ro;
    tbr_default_ransac_options(&ro);
    if (ransac_opt) ro = *ransac_opt;
    if (tbr_status c = check_ransac(ro)) return c;
    RunOptions o = make_run_options(&ro, nullptr, ext);
    std::vector<FrameHost> fr;
    for (int i = 0; i < n_frames; ++i) {
        if (tbr_status c = check_frame(frames[i])) return c;
        fr.push_back(frame_host(frames[i], ro));
    }
    return submit_frames(ctx, fr, o, false, nullptr, ticket);
}

tbr_status tbr_estimate_batch_device_submit(tbr_context *ctx, const tbr_frame_desc *frames, int32_t n_frames,
                                            const tbr_ransac_options *ransac_opt, const tbr_ext_options *ext,
                                            void *stream, tbr_ticket **ticket) {
    if (!ctx || !frames || n_frames < 1 || !ticket) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    *ticket = nullptr;
    if (n_frames > kMaxActive) return fail(TBR_ERR_INVALID_ARG, "more than 1024 frames in one submission");
    tbr_ransac_options ro;
    tbr_default_ransac_options(&ro);
    if (ransac_opt) ro = *ransac_opt;
    if (tbr_status c = check_ransac(ro)) return c;
    RunOptions o = make_run_options(&ro, nullptr, ext);
    std::vector<FrameHost> fr;
    if (tbr_status c = device_frames(ctx->E, frames, n_frames, ro, fr)) return c;
    return submit_frames(ctx, fr, o, true, stream, ticket);
}

tbr_status tbr_estimate_batch_collect(tbr_ticket *t, tbr_frame_result *results, uint8_t *const *inliers) {
    tbr_context *ctx = nullptr;
    {
        std::lock_guard<std::mutex> g(g_tickets_mu);
        auto it = t ? g_tickets.find(t) : g_tickets.end();
        if (it == g_tickets.end())
            return fail(TBR_ERR_INVALID_ARG, "unknown ticket (collected, or its context destroyed)");
        ctx = it->second;
        g_tickets.erase(it);
    }
    Engine &E = ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_ticket(t);
    tbr_status st = t->st;
    std::string msg = t->msg;
    const size_t n = t->slots.size();
    if (st == TBR_OK && inliers) {
        // On a stream of their own: the masks wait for nothing queued since.
        for (size_t i = 0; i < n && st == TBR_OK; ++i) {
            if (!inliers[i]) continue;
            const cudaError_t e = cudaMemcpyAsync(inliers[i], E.P.mask + t->devs[i].blk_off * kSub, t->ns[i],
                                                  cudaMemcpyDeviceToHost, E.stream_out);
            if (e != cudaSuccess) {
                st = TBR_ERR_CUDA;
                msg = std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e);
            }
        }
        const cudaError_t e = cudaStreamSynchronize(E.stream_out);
        if (st == TBR_OK && e != cudaSuccess) {
            st = TBR_ERR_CUDA;
            msg = std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e);
        }
    }
    if (st == TBR_OK && results)
        for (size_t i = 0; i < n; ++i) {
            for (int k = 0; k < 4; ++k) results[i].q[k] = t->res[i].q[k];
            for (int k = 0; k < 3; ++k) results[i].t[k] = t->res[i].t[k];
            results[i].status = TBR_OK;
            fill_stats(t->res[i], t->ns[i], &results[i].stats, t->ms);
        }
    release_frames(E, t->slots, t->devs);
    ctx->tickets.erase(std::find(ctx->tickets.begin(), ctx->tickets.end(), t));
    delete t;
    if (st) return fail(st, msg);
    return TBR_OK;
}

tbr_status tbr_get_inliers(tbr_context *ctx, const double q[4], const double t[3], const double *x,
                           const double *X, int64_t n, double sq_threshold, uint8_t *inliers,
                           int64_t *count) {
    if (!ctx || !q || !t || !x || !X || n < 0) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    Engine &E = ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(ctx);
    TBR_CUDA(cudaSetDevice(E.device));
    if (n == 0) {
        if (count) *count = 0;
        return TBR_OK;
    }
    const int64_t nb = (n + kSub - 1) / kSub;
    const int64_t off = E.blocks.alloc(nb);
    if (off < 0) return fail(TBR_ERR_OOM, "point workspace exhausted");
    const int64_t p0 = off * kSub;
    tbr_status st = E.ensure_stage(40 * n + 1024 + n);
    if (st) { E.blocks.release(off, nb); return st; }
    char *h = (char *)E.h_stage;
    std::memcpy(h, x, 16 * n);
    std::memcpy(h + 16 * n, X, 24 * n);
    double *hq = (double *)(h + 40 * n);
    for (int k = 0; k < 4; ++k) hq[k] = q[k];
    for (int k = 0; k < 3; ++k) hq[4 + k] = t[k];
    // x goes to the normalized-coordinate pool, X to the world-point pool; the
    // pose rides in the first hypothesis slot.
    TBR_CUDA(cudaMemcpyAsync(E.P.xn64 + 2 * p0, h, 16 * n, cudaMemcpyHostToDevice, E.stream));
    TBR_CUDA(cudaMemcpyAsync((void *)(E.P.X64 + 3 * p0), h + 16 * n, 24 * n, cudaMemcpyHostToDevice, E.stream));
    TBR_CUDA(cudaMemcpyAsync(E.P.hP64, hq, 7 * 8, cudaMemcpyHostToDevice, E.stream));
    TBR_CUDA(cudaMemsetAsync(E.P.counters + kCWorkPairs, 0, 8, E.stream));
    const int grid = (int)std::min<int64_t>(E.num_sms * 4, (n + 255) / 256);
    k_pose_mask<<<grid, 256, 0, E.stream>>>(E.P.xn64 + 2 * p0, E.P.X64 + 3 * p0, n, E.P.hP64, sq_threshold,
                                            E.P.mask + p0, E.P.counters + kCWorkPairs);
    st = TBR_OK;
    if (cudaGetLastError() != cudaSuccess) st = fail(TBR_ERR_CUDA, "k_pose_mask launch failed");
    uint8_t *hm = (uint8_t *)(h + 40 * n + 64);
    if (!st) {
        cudaMemcpyAsync(hm, E.P.mask + p0, n, cudaMemcpyDeviceToHost, E.stream);
        cudaMemcpyAsync(E.h_counters, E.P.counters, 8 * kCNum, cudaMemcpyDeviceToHost, E.stream);
    }
    if (cudaStreamSynchronize(E.stream) != cudaSuccess && !st) st = fail(TBR_ERR_CUDA, "get_inliers failed");
    E.blocks.release(off, nb);
    if (st) return st;
    if (inliers) std::memcpy(inliers, hm, n);
    if (count) *count = (int64_t)E.h_counters[kCWorkPairs];
    return TBR_OK;
}

tbr_status tbr_bundle_adjust(tbr_context *ctx, const double *x, const double *X, int64_t n, const double K[4],
                             double q[4], double t[3], const tbr_bundle_options *opt, const double *weights,
                             const tbr_ext_options *ext, tbr_stats *stats) {
    // The reference uses the Cauchy loss and unit weights whatever the options
    // (ba.cu:111-130, jaco.cuh:36,123); with honor_options the loss type and
    // the weights are applied.
    if (!ctx || !x || !X || !K || !q || !t || n < 0) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    if (!(K[0] > 0) || !(K[1] > 0)) return fail(TBR_ERR_INVALID_ARG, "focal lengths must be positive");
    tbr_bundle_options bo;
    tbr_default_bundle_options(&bo);
    if (opt) bo = *opt;
    if (!(bo.loss_scale > 0)) return fail(TBR_ERR_INVALID_ARG, "loss_scale must be > 0");
    const bool honor = ext && ext->honor_options;
    int32_t loss = kLossCauchy;
    if (honor) {
        switch (bo.loss_type) {  // BundleOptions_cuda::LossType, utils.h:45-52
            case 0: loss = kLossTrivial; break;
            case 1: loss = kLossTruncated; break;
            case 2: loss = kLossHuber; break;
            case 3: loss = kLossCauchy; break;
            default: return fail(TBR_ERR_INVALID_ARG, "loss type not supported (TRUNCATED_LE_ZACH)");
        }
    }
    const bool weighted = honor && weights != nullptr;
    Engine &E = ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(ctx);
    TBR_CUDA(cudaSetDevice(E.device));
    RunOptions o;
    FrameHost fh{x, X, std::max<int64_t>(n, 1), {K[0], K[1], K[2], K[3]}, 0, 1.0, nullptr, 0};
    if (n == 0) {
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return TBR_OK;
    }
    std::vector<int> slots;
    int64_t max_n = 0;
    TBR_CUDA(cudaMemsetAsync(E.P.counters, 0, 8 * kCNum, E.stream));
    tbr_status st = admit_frames(E, {fh}, o, slots, max_n);
    if (st) return st;
    FrameDev fd;
    TBR_CUDA(cudaMemcpyAsync(&fd, E.P.frames + slots[0], sizeof(FrameDev), cudaMemcpyDeviceToHost, E.stream));
    TBR_CUDA(cudaStreamSynchronize(E.stream));
    fd.status = kLMPending;
    fd.lm_force_cluster = 1;
    fd.focal = 1.0;
    for (int k = 0; k < 4; ++k) fd.lm_cam[k] = K[k];
    fd.lm_inv_sq_thr = 1.0 / (bo.loss_scale * bo.loss_scale);  // CauchyLoss_cuda(loss_scale)
    fd.lm_thr = bo.loss_scale;
    fd.lm_loss = loss;
    fd.lm_weighted = weighted ? 1 : 0;
    if (weighted)
        TBR_CUDA(cudaMemcpyAsync(E.P.lw64 + fd.blk_off * kSub, weights, 8 * n, cudaMemcpyHostToDevice, E.stream));
    fd.lm_max_iter = (int64_t)bo.max_iterations;
    fd.lm_grad_tol = bo.gradient_tol;
    fd.lm_step_tol = bo.step_tol;
    fd.lm_lambda0 = bo.initial_lambda;
    fd.lm_min_lambda = bo.min_lambda;
    fd.lm_max_lambda = bo.max_lambda;
    fd.skip_refine = 0;
    FrameResult r0;
    std::memset(&r0, 0, sizeof(r0));
    for (int k = 0; k < 4; ++k) r0.q[k] = q[k];
    for (int k = 0; k < 3; ++k) r0.t[k] = t[k];
    TBR_CUDA(cudaMemcpyAsync(E.P.frames + slots[0], &fd, sizeof(FrameDev), cudaMemcpyHostToDevice, E.stream));
    TBR_CUDA(cudaMemcpyAsync(E.P.results + slots[0], &r0, sizeof(FrameResult), cudaMemcpyHostToDevice, E.stream));
    const int bx = (int)std::min<int64_t>(64, std::max<int64_t>(1, (n + 1023) / 1024));
    k_prep_bounds<<<dim3(bx, 1), 256, 0, E.stream>>>(E.P);
    k_lm_pack<<<bx, 256, 0, E.stream>>>(E.P);
    cudaEventRecord(E.ev0, E.stream);
    k_lm<<<kLMCluster, kLMThreads, 0, E.stream>>>(E.P);
    cudaEventRecord(E.ev1, E.stream);
    st = TBR_OK;
    if (cudaGetLastError() != cudaSuccess) st = fail(TBR_ERR_CUDA, "bundle_adjust launch failed");
    FrameResult res;
    if (!st) cudaMemcpyAsync(&res, E.P.results + slots[0], sizeof(FrameResult), cudaMemcpyDeviceToHost, E.stream);
    if (cudaStreamSynchronize(E.stream) != cudaSuccess && !st) st = fail(TBR_ERR_CUDA, "bundle_adjust failed");
    E.blocks.release(fd.blk_off, fd.n_blocks);
    E.free_slots.push_back(slots[0]);
    if (st) return st;
    for (int k = 0; k < 4; ++k) q[k] = res.q[k];
    for (int k = 0; k < 3; ++k) t[k] = res.t[k];
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, E.ev0, E.ev1);
        stats->gpu_ms = ms;
        stats->lm_iterations = res.lm_iters;
        stats->lm_invalid_steps = res.lm_invalid;
        stats->lm_initial_cost = res.lm_cost0;
        stats->lm_cost = res.lm_cost;
    }
    return TBR_OK;
}

}  // extern "C"

// --------------------------------------------------------------- batches --
struct tbr_batch {
    tbr_context *ctx = nullptr;
    std::vector<int> slots;
    std::vector<int64_t> ns, blk_off, n_blocks;
    RunOptions o;
    Pools Q{};
    int32_t *d_active = nullptr;
    FrameDev *d_init = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    bool launched = false;
    Engine::Profile prof;
};

// Live batches. Destroying a context frees the batches made on it; their
// handles then stay known as dead, so that a later call on one is refused
// instead of touching freed memory.
static std::mutex g_batches_mu;
static std::unordered_map<tbr_batch *, tbr_context *> g_batches;

static bool live_batch(tbr_batch *b) {
    std::lock_guard<std::mutex> lk(g_batches_mu);
    return b && g_batches.count(b) != 0;
}

static void batch_free(tbr_batch *b) {
    if (!b) return;
    Engine &E = b->ctx->E;
    cudaStreamSynchronize(E.stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->d_active) cudaFree(b->d_active);
    if (b->d_init) cudaFree(b->d_init);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    for (auto &e : b->prof.ev)
        if (e) cudaEventDestroy(e);
    for (size_t i = 0; i < b->slots.size(); ++i) {
        if (i < b->blk_off.size()) E.blocks.release(b->blk_off[i], b->n_blocks[i]);
        E.free_slots.push_back(b->slots[i]);
    }
    delete b;
}

static void destroy_context_batches(tbr_context *ctx) {
    std::vector<tbr_batch *> mine;
    {
        std::lock_guard<std::mutex> lk(g_batches_mu);
        for (auto it = g_batches.begin(); it != g_batches.end();) {
            if (it->second == ctx) {
                mine.push_back(it->first);
                it = g_batches.erase(it);
            } else {
                ++it;
            }
        }
    }
    std::lock_guard<std::mutex> lk(ctx->E.mu);
    for (tbr_batch *b : mine) batch_free(b);
}

extern "C" {

tbr_status tbr_batch_create(tbr_context *ctx, const tbr_frame_desc *frames, int32_t n_frames,
                            const tbr_ransac_options *ransac_opt, const tbr_ext_options *ext, tbr_batch **out) {
    if (!ctx || !frames || n_frames < 1 || !out) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    if (n_frames > kMaxActive) return fail(TBR_ERR_INVALID_ARG, "at most 1024 frames per batch");
    tbr_ransac_options ro;
    tbr_default_ransac_options(&ro);
    if (ransac_opt) ro = *ransac_opt;
    if (tbr_status c = check_ransac(ro)) return c;
    std::vector<FrameHost> fr;
    for (int i = 0; i < n_frames; ++i) {
        if (tbr_status c = check_frame(frames[i])) return c;
        fr.push_back(frame_host(frames[i], ro));
    }
    Engine &E = ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(ctx);
    TBR_CUDA(cudaSetDevice(E.device));
    auto *b = new tbr_batch();
    b->ctx = ctx;
    b->o = make_run_options(&ro, nullptr, ext);
    int64_t max_n = 0;
    std::vector<FrameDev> devs;
    tbr_status st = admit_frames(E, fr, b->o, b->slots, max_n, &devs);
    for (size_t i = 0; i < b->slots.size() && i < devs.size(); ++i) {  // what batch_free releases
        b->ns.push_back(devs[i].n);
        b->blk_off.push_back(devs[i].blk_off);
        b->n_blocks.push_back(devs[i].n_blocks);
    }
    if (st) {
        batch_free(b);
        return st;
    }
    // The batch keeps its own active list so that other calls on the context
    // can run between its launches.
    if (cudaMalloc(&b->d_active, 4 * n_frames) != cudaSuccess ||
        cudaMalloc(&b->d_init, sizeof(FrameDev) * n_frames) != cudaSuccess) {
        batch_free(b);
        return fail(TBR_ERR_OOM, "batch allocation failed");
    }
    cudaMemcpyAsync(b->d_active, E.d_active, 4 * n_frames, cudaMemcpyDeviceToDevice, E.stream);
    b->Q = E.P;
    b->Q.active = b->d_active;
    b->Q.n_active = n_frames;
    E.launch_prep(b->Q, n_frames, max_n);
    // Snapshot the prepared frame states (AABB centre included).
    for (int i = 0; i < n_frames; ++i)
        cudaMemcpyAsync(b->d_init + i, E.P.frames + b->slots[i], sizeof(FrameDev), cudaMemcpyDeviceToDevice, E.stream);
    if (cudaStreamSynchronize(E.stream) != cudaSuccess) {
        batch_free(b);
        return fail(TBR_ERR_CUDA, "batch upload failed");
    }
    E.pp = b->o.pp;
    bool ok = E.build_loop_graph(b->Q, n_frames, b->o.hr, b->d_init, &b->graph, &b->exec);
    if (ok) ok = cudaEventCreate(&b->e0) == cudaSuccess && cudaEventCreate(&b->e1) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        batch_free(b);
        return fail(TBR_ERR_CUDA, "graph capture failed");
    }
    {
        std::lock_guard<std::mutex> lk(g_batches_mu);
        g_batches[b] = ctx;
    }
    *out = b;
    return TBR_OK;
}

tbr_status tbr_batch_autotune(tbr_batch *b, int32_t repeats, tbr_tune_entry *entries, int32_t max,
                              int32_t *n_out, tbr_tune_entry *best) {
    if (!live_batch(b) || repeats < 1 || max < 0) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    Engine &E = b->ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(b->ctx);
    TBR_CUDA(cudaSetDevice(E.device));
    const int n = (int)b->slots.size();
    struct Shape {
        int hr, pp;
    };
    // Hypotheses per block x point tile per work item: 32 (the tensor-core
    // kernel) and 64 / 128 / 192 / 256 (the compiled FP32 variants, 2 / 4 / 6 / 8
    // per lane, with 2 or 4 points per inner step) x tiles of 128, 256 and 512
    // points, plus tiles sized from the step's work (0) and longer ones.
    const Shape shapes[6] = {{2, 4}, {4, 2}, {4, 4}, {6, 2}, {6, 4}, {8, 2}};
    const int chunks[6] = {0, 128, 256, 512, 1024, 2048};
    const int tc_chunks[5] = {0, 128, 256, 512, 8192};
    struct Cand {
        int hr, pp, chunk;
    };
    std::vector<Cand> cands;
    for (const Shape &sh : shapes)
        for (int chunk : chunks) cands.push_back({sh.hr, sh.pp, chunk});
    for (int chunk : tc_chunks) cands.push_back({1, kTcPP, chunk});
    std::vector<tbr_tune_entry> tried;
    cudaEvent_t t0, t1;
    TBR_CUDA(cudaEventCreate(&t0));
    TBR_CUDA(cudaEventCreate(&t1));
    auto apply = [&](int hr, int pp, int chunk, cudaGraph_t *g, cudaGraphExec_t *x) -> bool {
        k_set_shape<<<(n + 127) / 128, 128, 0, E.stream>>>(b->d_init, n, hr, chunk);
        if (cudaGetLastError() != cudaSuccess) return false;
        E.pp = pp;
        return E.build_loop_graph(b->Q, n, hr, b->d_init, g, x);
    };
    tbr_status st = TBR_OK;
    for (const Cand &cd : cands) {
        {
            cudaGraph_t g = nullptr;
            cudaGraphExec_t x = nullptr;
            if (!apply(cd.hr, cd.pp, cd.chunk, &g, &x)) {
                st = fail(TBR_ERR_CUDA, "autotune graph capture failed");
                break;
            }
            float ms = 0.f;
            cudaError_t e = cudaGraphLaunch(x, E.stream);  // warm-up
            if (e == cudaSuccess) e = cudaEventRecord(t0, E.stream);
            for (int r = 0; r < repeats && e == cudaSuccess; ++r) e = cudaGraphLaunch(x, E.stream);
            if (e == cudaSuccess) e = cudaEventRecord(t1, E.stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(t1);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
            cudaGraphExecDestroy(x);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                st = fail(TBR_ERR_CUDA, cudaGetErrorString(e));
                break;
            }
            TBR_CUDA(cudaMemcpy(E.h_counters, b->Q.counters, 8 * kCNum, cudaMemcpyDeviceToHost));
            if (E.h_counters[kCError]) {
                st = fail(TBR_ERR_INTERNAL, "device error during autotune");
                break;
            }
            tried.push_back({cd.hr, cd.pp, cd.chunk, 0, (double)ms / repeats});
        }
        if (st) break;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (st) return st;
    size_t bi = 0;
    for (size_t i = 1; i < tried.size(); ++i)
        if (tried[i].ms < tried[bi].ms) bi = i;
    const tbr_tune_entry win = tried[bi];
    // Keep the winner: new initial records and graph for tbr_batch_run.
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    if (!apply(win.hyp_per_thread, win.points_per_iter, win.chunk_points, &g, &x))
        return fail(TBR_ERR_CUDA, "autotune graph capture failed");
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph = g;
    b->exec = x;
    b->o.hr = win.hyp_per_thread;
    b->o.pp = win.points_per_iter;
    b->o.chunk_points = win.chunk_points;
    b->launched = false;
    TBR_CUDA(cudaStreamSynchronize(E.stream));
    if (entries)
        for (int i = 0; i < (int)tried.size() && i < max; ++i) entries[i] = tried[i];
    if (n_out) *n_out = (int32_t)tried.size();
    if (best) *best = win;
    return TBR_OK;
}

tbr_status tbr_batch_run(tbr_batch *b) {
    if (!live_batch(b)) return fail(TBR_ERR_INVALID_ARG, "NULL or destroyed batch");
    Engine &E = b->ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(b->ctx);
    TBR_CUDA(cudaSetDevice(E.device));
    TBR_CUDA(cudaEventRecord(b->e0, E.stream));
    TBR_CUDA(cudaGraphLaunch(b->exec, E.stream));
    TBR_CUDA(cudaEventRecord(b->e1, E.stream));
    b->launched = true;
    return TBR_OK;
}

tbr_status tbr_batch_sync(tbr_batch *b) {
    if (!live_batch(b)) return fail(TBR_ERR_INVALID_ARG, "NULL or destroyed batch");
    Engine &E = b->ctx->E;
    TBR_CUDA(cudaStreamSynchronize(E.stream));
    TBR_CUDA(cudaMemcpy(E.h_counters, b->Q.counters, 8 * kCNum, cudaMemcpyDeviceToHost));
    if (E.h_counters[kCError] & kErrTimeout) return fail(TBR_ERR_TIMEOUT, "bounded device wait expired");
    if (E.h_counters[kCError] & kErrOverflow) return fail(TBR_ERR_INTERNAL, "step limit or capacity exceeded");
    return TBR_OK;
}

tbr_status tbr_batch_results(tbr_batch *b, tbr_frame_result *results) {
    if (!live_batch(b) || !results) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    Engine &E = b->ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(b->ctx);
    TBR_CUDA(cudaStreamSynchronize(E.stream));
    float ms = 0.f;
    if (b->launched) cudaEventElapsedTime(&ms, b->e0, b->e1);
    std::vector<FrameResult> r(b->slots.size());
    tbr_status st = fetch_results(E, b->slots, r.data());
    if (st) return st;
    for (size_t i = 0; i < b->slots.size(); ++i) {
        for (int k = 0; k < 4; ++k) results[i].q[k] = r[i].q[k];
        for (int k = 0; k < 3; ++k) results[i].t[k] = r[i].t[k];
        results[i].status = r[i].status == kDone ? TBR_OK : TBR_ERR_INTERNAL;
        fill_stats(r[i], b->ns[i], &results[i].stats, ms);
    }
    return TBR_OK;
}

tbr_status tbr_batch_profile(tbr_batch *b, tbr_kernel_profile *out, int32_t max, int32_t *n_out,
                             uint64_t *pairs_scored) {
    if (!live_batch(b) || !out) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    Engine &E = b->ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(b->ctx);
    TBR_CUDA(cudaSetDevice(E.device));
    Engine::Profile pr;
    k_reset_frames<<<b->Q.n_active, 128, 0, E.stream>>>(b->Q, b->d_init);
    int steps = 0;
    E.pp = b->o.pp;
    tbr_status st = E.run(b->Q, b->Q.n_active, b->o.hr, 100000, &steps, &pr);
    for (auto &e : pr.ev)
        if (e) cudaEventDestroy(e);
    if (st) return st;
    if (pairs_scored) *pairs_scored = E.h_counters[kCPairsTotal];
    int m = 0;
    for (int k = 0; k < 10 && m < max; ++k, ++m) {
        std::snprintf(out[m].name, sizeof(out[m].name), "%s", Engine::kKernelNames[k]);
        out[m].total_ms = pr.ms[k];
        out[m].launches = pr.launches[k];
    }
    if (n_out) *n_out = m;
    return TBR_OK;
}

tbr_status tbr_measure_fp32_peak(tbr_context *ctx, double *tflops) {
    if (!ctx || !tflops) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    Engine &E = ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(ctx);
    TBR_CUDA(cudaSetDevice(E.device));
    const int blocks = E.num_sms * 8, threads = 256, iters = 1 << 14;
    float *sink = (float *)E.P.hS32;  // never written (see k_fp32_peak)
    k_fp32_peak<<<blocks, threads, 0, E.stream>>>(sink, 256, 0.999f, 1e-3f);  // warm-up
    TBR_CUDA(cudaEventRecord(E.ev0, E.stream));
    for (int r = 0; r < 4; ++r) k_fp32_peak<<<blocks, threads, 0, E.stream>>>(sink, iters, 0.999f, 1e-3f);
    TBR_CUDA(cudaEventRecord(E.ev1, E.stream));
    TBR_CUDA(cudaEventSynchronize(E.ev1));
    float ms = 0.f;
    TBR_CUDA(cudaEventElapsedTime(&ms, E.ev0, E.ev1));
    const double flop = 4.0 * blocks * threads * (double)iters * 8 * 4;  // 8 f32x2 FMA = 32 FLOP
    *tflops = flop / (ms * 1e-3) / 1e12;
    return TBR_OK;
}

void tbr_batch_destroy(tbr_batch *b) {
    {
        // (the handle is erased first: a concurrent tbr_context_destroy then skips it)
        std::lock_guard<std::mutex> lk(g_batches_mu);
        if (!b || !g_batches.erase(b)) return;  // NULL, or already freed with its context
    }
    std::lock_guard<std::mutex> lk(b->ctx->E.mu);
    retire_tickets(b->ctx);
    batch_free(b);
}

}  // extern "C"

// --------------------------------------------------------------- serving --
// Continuous batching. A worker thread owns a dedicated Engine sized by the
// workspace budget and loops:
//   1. retire: frames whose LM finished -> results out, slot and blocks freed;
//   2. admit: queued requests, in arrival order, while a slot and point blocks
//      are free (the budget is the engine workspace), uploaded and prepared;
//   3. one engine step over every resident frame (RANSAC of the frames still
//      sampling, inliers + LM of the frames that finished).
// A request that arrives while others run therefore joins the next step and
// its work overlaps theirs on the device.
struct ServerRequest {
    uint64_t id;
    std::vector<double> uv, xyz;            // owned copies (tbr_server_submit)
    const double *ext_uv = nullptr, *ext_xyz = nullptr;  // caller's arrays (tbr_server_submit_nocopy)
    int64_t n = 0;
    double K[4];
    uint64_t seed;
    double thr;
    std::chrono::steady_clock::time_point t_submit;
    bool cancelled = false;
    const double *U() const { return ext_uv ? ext_uv : uv.data(); }
    const double *Xw() const { return ext_xyz ? ext_xyz : xyz.data(); }
};

struct Resident {
    std::unique_ptr<ServerRequest> req;
    int slot;
    int64_t blk_off, n_blocks;
};

struct PinnedBuffer {
    void *p = nullptr;
    size_t bytes = 0;
    // Grows geometrically: pinning is slow and freeing pinned memory
    // synchronizes the device.
    tbr_status ensure(size_t b) {
        if (b <= bytes) return TBR_OK;
        const size_t nb = std::max(b, 2 * bytes);
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        TBR_CUDA(cudaMallocHost(&p, nb));
        bytes = nb;
        return TBR_OK;
    }
    ~PinnedBuffer() {
        if (p) cudaFreeHost(p);
    }
};

struct tbr_server {
    Engine E;
    RunOptions o;
    tbr_ransac_options ro;
    int max_queue = 1 << 16;
    std::mutex mu;
    std::condition_variable cv, cv_done;
    std::deque<std::unique_ptr<ServerRequest>> queue;
    std::vector<Resident> resident;
    std::vector<tbr_server_result> done;
    std::vector<uint64_t> cancel_ids;
    uint64_t next_id = 1;
    uint64_t in_flight = 0;  // submitted and not yet completed
    bool stop = false;
    std::thread worker;
    int32_t *d_status = nullptr, *d_prep = nullptr;
    // Host side of the steps in flight (at most two), per buffer b: the
    // resident frames' statuses and results at the end of the step (pinned),
    // its counters, its active list, and an event after its downloads.
    int32_t *h_status[2] = {}, *h_active[2] = {};
    FrameResult *h_res[2] = {};
    unsigned long long *h_cnt[2] = {};
    cudaEvent_t ev_done[2] = {};
    struct InFlight {
        int buf;                     // host buffers b
        int stage;                   // admission staging buffer it uploads from (-1: none)
        std::vector<uint64_t> ids;   // request ids in active-list order
    };
    std::deque<InFlight> inflight;
    PinnedBuffer stage[2];   // admission staging; a step in flight holds the one it uploads from
    tbr_server_stats stats{};  // guarded by mu
    tbr_server_stats ws{};     // the worker's own counters, published into stats after each step
    tbr_status error = TBR_OK;
    std::string error_msg;
};

static double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

static void server_complete(tbr_server *s, Resident &r, const FrameResult *res, tbr_status st) {
    tbr_server_result out;
    std::memset(&out, 0, sizeof(out));
    out.request_id = r.req->id;
    out.status = st;
    if (res) {
        for (int k = 0; k < 4; ++k) out.q[k] = res->q[k];
        for (int k = 0; k < 3; ++k) out.t[k] = res->t[k];
        fill_stats(*res, r.req->n, &out.stats, 0.f);
    }
    out.submit_to_done_ms = ms_since(r.req->t_submit);
    std::lock_guard<std::mutex> lk(s->mu);
    s->done.push_back(out);
    s->in_flight--;
    s->stats.completed++;
    s->cv_done.notify_all();
}

// Resident frames from which a serving step overlaps refinement with RANSAC,
// and from which the loop keeps a second step queued on the device.
constexpr int kServerOverlapFrames = 16;

// Retires the oldest step in flight: waits for it, then completes the frames it
// finished that are still resident (a frame that finished earlier may show up
// again in a later step's snapshot, which was taken before its retirement).
static tbr_status server_retire_oldest(tbr_server *s) {
    Engine &E = s->E;
    tbr_server::InFlight st = std::move(s->inflight.front());
    s->inflight.pop_front();
    auto t0 = std::chrono::steady_clock::now();
    TBR_CUDA(cudaEventSynchronize(s->ev_done[st.buf]));
    s->ws.device_wait_ms += ms_since(t0);
    if (s->h_cnt[st.buf][kCError] & kErrTimeout) return fail(TBR_ERR_TIMEOUT, "bounded device wait expired");
    s->ws.pairs_scored = (int64_t)s->h_cnt[st.buf][kCPairsTotal];
    t0 = std::chrono::steady_clock::now();
    std::unordered_map<uint64_t, size_t> pos;
    for (size_t i = 0; i < s->resident.size(); ++i) pos[s->resident[i].req->id] = i;
    std::vector<bool> gone(s->resident.size(), false);
    bool any = false;
    for (size_t i = 0; i < st.ids.size(); ++i) {
        if (s->h_status[st.buf][i] != kDone) continue;
        auto it = pos.find(st.ids[i]);
        if (it == pos.end() || gone[it->second]) continue;  // retired or cancelled already
        Resident &r = s->resident[it->second];
        server_complete(s, r, &s->h_res[st.buf][i], TBR_OK);
        E.blocks.release(r.blk_off, r.n_blocks);
        E.free_slots.push_back(r.slot);
        gone[it->second] = true;
        any = true;
    }
    if (any) {
        std::vector<Resident> keep;
        for (size_t i = 0; i < s->resident.size(); ++i)
            if (!gone[i]) keep.push_back(std::move(s->resident[i]));
        s->resident.swap(keep);
    }
    s->ws.host_retire_ms += ms_since(t0);
    return TBR_OK;
}

// One iteration of the request loop, pipelined with the device. With many
// resident frames two steps are kept in flight, so the device always has a
// queued step while the host retires, stages and launches:
//   1. if two steps are in flight, retire the older one;
//   2. take queued requests that fit the free slots and point blocks and copy
//      them into a staging buffer no step in flight uploads from;
//   3. with few resident frames (latency first) retire the step in flight too;
//   4. upload the staged frames, prepare them, and launch the next step over
//      every resident frame without waiting for it.
// Device writes of a new step (records, points) are ordered after the steps in
// flight on the one stream, so a slot or block freed by a retirement can be
// reused at once.
static tbr_status server_step(tbr_server *s) {
    Engine &E = s->E;
    while (s->inflight.size() >= 2) {
        tbr_status st = server_retire_oldest(s);
        if (st) return st;
    }
    // ---- stage admissions ----
    auto t0 = std::chrono::steady_clock::now();
    int sb = 0;
    for (auto &f : s->inflight)
        if (f.stage == sb) sb = 1;
    std::vector<std::unique_ptr<ServerRequest>> newreq;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        int64_t free_blocks = E.blocks.capacity() - E.blocks.used();
        // One step admits at most a staging buffer's worth (always at least one
        // request), so that staging keeps overlapping the device's steps.
        size_t staged = 0;
        const size_t stage_cap = s->stage[sb].bytes;
        while (!s->queue.empty() && (int)newreq.size() < (int)E.free_slots.size()) {
            auto &q = s->queue.front();
            if (q->cancelled) {
                tbr_server_result o;
                std::memset(&o, 0, sizeof(o));
                o.request_id = q->id;
                o.status = TBR_ERR_CANCELLED;
                s->done.push_back(o);
                s->queue.pop_front();
                s->in_flight--;
                s->cv_done.notify_all();
                continue;
            }
            const int64_t need = (q->n + kSub - 1) / kSub;
            if (free_blocks < need) break;  // budget: wait for frames to retire
            const size_t bytes = (size_t)need * kSub * 40 + 2 * sizeof(FrameDev) + 1024;
            if (!newreq.empty() && staged + bytes > stage_cap) break;
            staged += bytes;
            free_blocks -= need;
            newreq.push_back(std::move(q));
            s->queue.pop_front();
        }
    }
    StagedAdmission A;
    if (!newreq.empty()) {
        std::vector<FrameHost> fh;
        for (auto &r : newreq)
            fh.push_back({r->U(), r->Xw(), r->n, {r->K[0], r->K[1], r->K[2], r->K[3]}, r->seed, r->thr, nullptr, 0});
        PinnedBuffer &buf = s->stage[sb];
        tbr_status st = buf.ensure(stage_bytes(fh));
        if (st) return st;
        st = stage_frames(E, fh, s->o, (char *)buf.p, A);
        if (st == TBR_ERR_OOM) {  // fragmentation: requeue at the front and retry after retirements
            std::lock_guard<std::mutex> lk(s->mu);
            for (auto it = newreq.rbegin(); it != newreq.rend(); ++it) s->queue.push_front(std::move(*it));
            newreq.clear();
        } else if (st) {
            return st;
        }
    }
    s->ws.host_stage_ms += ms_since(t0);
    // ---- few (or no) resident frames: finish the step in flight first ----
    const size_t will_resident = s->resident.size() + A.slots.size();
    if (!s->inflight.empty() && will_resident < (size_t)kServerOverlapFrames) {
        tbr_status st = server_retire_oldest(s);
        if (st) return st;
    }
    // ---- cancels of resident frames ----
    {
        std::vector<uint64_t> ids;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            ids.swap(s->cancel_ids);
        }
        for (uint64_t id : ids)
            for (size_t i = 0; i < s->resident.size(); ++i)
                if (s->resident[i].req->id == id) {
                    server_complete(s, s->resident[i], nullptr, TBR_ERR_CANCELLED);
                    E.blocks.release(s->resident[i].blk_off, s->resident[i].n_blocks);
                    E.free_slots.push_back(s->resident[i].slot);
                    s->resident.erase(s->resident.begin() + i);
                    break;
                }
    }
    // ---- upload admissions, launch the next step ----
    t0 = std::chrono::steady_clock::now();
    if (!A.slots.empty()) {
        tbr_status st = upload_staged(E, A);
        if (st) return st;
        // upload_staged wrote the new slots to d_active; prepare them (AABB, packing).
        TBR_CUDA(cudaMemcpyAsync(s->d_prep, E.d_active, 4 * A.slots.size(), cudaMemcpyDeviceToDevice, E.stream));
        Pools Q = E.P;
        Q.active = s->d_prep;
        Q.n_active = (int32_t)A.slots.size();
        E.launch_prep(Q, (int)A.slots.size(), A.max_n);
        for (size_t i = 0; i < A.slots.size(); ++i)
            s->resident.push_back({std::move(newreq[i]), A.slots[i], A.devs[i].blk_off, A.devs[i].n_blocks});
        s->ws.admitted += (int64_t)A.slots.size();
    }
    if (!s->resident.empty()) {
        const int na = (int)s->resident.size();
        int b = 0;
        for (auto &f : s->inflight)
            if (f.buf == b) b = 1;
        int32_t *ha = s->h_active[b];
        tbr_server::InFlight fl;
        fl.buf = b;
        fl.stage = A.slots.empty() ? -1 : sb;
        fl.ids.resize(na);
        for (int i = 0; i < na; ++i) {
            ha[i] = s->resident[i].slot;
            fl.ids[i] = s->resident[i].req->id;
        }
        TBR_CUDA(cudaMemcpyAsync(E.d_active, ha, 4 * na, cudaMemcpyHostToDevice, E.stream));
        E.P.n_active = na;
        if (na >= kServerOverlapFrames) {
            // Many resident frames: the refinement of frames that finished RANSAC
            // in earlier steps runs beside this step's RANSAC (disjoint frames);
            // a frame is refined one step after it finishes (a stream of requests
            // has no last step to defer it to, unlike a batch).
            TBR_CUDA(cudaEventRecord(E.ev_fork, E.stream));
            TBR_CUDA(cudaStreamWaitEvent(E.stream2, E.ev_fork, 0));
            E.launch_refine(E.P, na, E.stream2);
            E.launch_ransac(E.P, na, s->o.hr, E.stream);
            TBR_CUDA(cudaEventRecord(E.ev_join, E.stream2));
            TBR_CUDA(cudaStreamWaitEvent(E.stream, E.ev_join, 0));
            k_tick<<<1, 1, 0, E.stream>>>(E.P);
        } else {
            // Few: RANSAC, then the refinement of what finished, in this step
            // (each frame's LM on a CTA or a cluster, for latency).
            Pools Ql = E.P;
            Ql.lm_cluster_min = kLMClusterMinTail;
            E.launch_step(Ql, na, s->o.hr);
        }
        k_gather_status<<<(na + 255) / 256, 256, 0, E.stream>>>(E.P, s->d_status);
        k_gather_results<<<(int)std::min<size_t>(1024, (na * (sizeof(FrameResult) / 8) + 255) / 256), 256, 0,
                           E.stream>>>(E.P.results, E.d_active, na, E.d_res_stage);
        TBR_CUDA(cudaGetLastError());
        TBR_CUDA(cudaMemcpyAsync(s->h_status[b], s->d_status, 4 * na, cudaMemcpyDeviceToHost, E.stream));
        TBR_CUDA(cudaMemcpyAsync(s->h_res[b], E.d_res_stage, sizeof(FrameResult) * na, cudaMemcpyDeviceToHost,
                                 E.stream));
        TBR_CUDA(cudaMemcpyAsync(s->h_cnt[b], E.P.counters, 8 * kCNum, cudaMemcpyDeviceToHost, E.stream));
        TBR_CUDA(cudaEventRecord(s->ev_done[b], E.stream));
        s->inflight.push_back(std::move(fl));
        s->ws.steps++;
        s->ws.resident_sum += na;
    }
    s->ws.host_launch_ms += ms_since(t0);
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.steps = s->ws.steps;
    s->stats.admitted = s->ws.admitted;
    s->stats.resident_sum = s->ws.resident_sum;
    s->stats.host_stage_ms = s->ws.host_stage_ms;
    s->stats.device_wait_ms = s->ws.device_wait_ms;
    s->stats.host_retire_ms = s->ws.host_retire_ms;
    s->stats.host_launch_ms = s->ws.host_launch_ms;
    s->stats.pairs_scored = s->ws.pairs_scored;
    return TBR_OK;
}

static void server_loop(tbr_server *s) {
    cudaSetDevice(s->E.device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait_for(lk, std::chrono::milliseconds(50), [&] {
                return s->stop || !s->queue.empty() || !s->resident.empty() || !s->inflight.empty() ||
                       !s->cancel_ids.empty();
            });
            if (s->stop) break;
            if (s->queue.empty() && s->resident.empty() && s->inflight.empty()) {
                s->cancel_ids.clear();  // nothing resident to cancel
                continue;
            }
        }
        tbr_status st = server_step(s);
        if (st) {
            cudaStreamSynchronize(s->E.stream);
            s->inflight.clear();
            std::lock_guard<std::mutex> lk(s->mu);
            s->error = st;
            s->error_msg = g_last_error;
            // fail everything outstanding
            for (auto &r : s->resident) {
                tbr_server_result o;
                std::memset(&o, 0, sizeof(o));
                o.request_id = r.req->id;
                o.status = st;
                s->done.push_back(o);
            }
            for (auto &q : s->queue) {
                tbr_server_result o;
                std::memset(&o, 0, sizeof(o));
                o.request_id = q->id;
                o.status = st;
                s->done.push_back(o);
            }
            s->in_flight = 0;
            s->resident.clear();
            s->queue.clear();
            s->cv_done.notify_all();
            break;
        }
    }
    cudaStreamSynchronize(s->E.stream);
}

static void server_free(tbr_server *s) {
    if (s->d_status) cudaFree(s->d_status);
    if (s->d_prep) cudaFree(s->d_prep);
    for (int b = 0; b < 2; ++b) {
        if (s->h_status[b]) cudaFreeHost(s->h_status[b]);
        if (s->h_active[b]) cudaFreeHost(s->h_active[b]);
        if (s->h_res[b]) cudaFreeHost(s->h_res[b]);
        if (s->h_cnt[b]) cudaFreeHost(s->h_cnt[b]);
        if (s->ev_done[b]) cudaEventDestroy(s->ev_done[b]);
    }
    delete s;
}

extern "C" {

tbr_status tbr_server_create(tbr_context *ctx, const tbr_server_config *cfg, tbr_server **out) {
    if (!ctx || !cfg || !out) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    auto *s = new tbr_server();
    const uint64_t budget = cfg->workspace_budget_bytes ? cfg->workspace_budget_bytes : (8ull << 30);
    const int slots = cfg->max_slots > 0 ? std::min(cfg->max_slots, kMaxActive) : 512;
    tbr_status st = s->E.init(ctx->E.device, budget, slots);
    if (st) {
        delete s;
        return st;
    }
    s->ro = cfg->ransac;
    if (tbr_status c = check_ransac(s->ro)) {
        delete s;
        return c;
    }
    s->o = make_run_options(&s->ro, nullptr, &cfg->ext);
    // Serving: bounded rounds per step so that one heavy frame cannot hold a
    // step (and the requests arriving meanwhile) for long.
    s->o.max_rounds_step = 64;
    s->E.pp = s->o.pp;
    if (cfg->max_queue > 0) s->max_queue = cfg->max_queue;
    bool ok = cudaMalloc(&s->d_status, 4 * kMaxActive) == cudaSuccess &&
              cudaMalloc(&s->d_prep, 4 * kMaxActive) == cudaSuccess;
    for (int b = 0; b < 2 && ok; ++b)
        ok = cudaMallocHost(&s->h_status[b], 4 * kMaxActive) == cudaSuccess &&
             cudaMallocHost(&s->h_active[b], 4 * kMaxActive) == cudaSuccess &&
             cudaMallocHost(&s->h_res[b], sizeof(FrameResult) * kMaxActive) == cudaSuccess &&
             cudaMallocHost(&s->h_cnt[b], 8 * kCNum) == cudaSuccess &&
             cudaEventCreateWithFlags(&s->ev_done[b], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        server_free(s);
        return fail(TBR_ERR_OOM, "server allocation failed");
    }
    // Staging for one step's admissions, sized up front (128 MiB each).
    for (auto &b : s->stage)
        if (b.ensure(128ull << 20) != TBR_OK) {
            server_free(s);
            return fail(TBR_ERR_OOM, "server staging allocation failed");
        }
    if (s->E.ensure_stage(1 << 20) != TBR_OK) {
        server_free(s);
        return fail(TBR_ERR_OOM, "server staging allocation failed");
    }
    cudaMemsetAsync(s->E.P.counters, 0, 8 * kCNum, s->E.stream);
    cudaStreamSynchronize(s->E.stream);
    s->worker = std::thread(server_loop, s);
    *out = s;
    return TBR_OK;
}

static tbr_status server_enqueue(tbr_server *s, std::unique_ptr<ServerRequest> r, const tbr_frame_desc *frame,
                                 uint64_t *request_id) {
    r->n = frame->n;
    for (int k = 0; k < 4; ++k) r->K[k] = frame->K[k];
    r->seed = frame->seed;
    r->thr = frame->max_reproj_error > 0 ? frame->max_reproj_error : s->ro.max_reproj_error;
    r->t_submit = std::chrono::steady_clock::now();
    if ((frame->n + kSub - 1) / kSub > s->E.blocks.capacity())
        return fail(TBR_ERR_CAPACITY, "frame larger than the serving budget");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->error) return fail(s->error, s->error_msg);
    if ((int)s->queue.size() >= s->max_queue) return fail(TBR_ERR_CAPACITY, "queue full");
    r->id = s->next_id++;
    if (request_id) *request_id = r->id;
    s->queue.push_back(std::move(r));
    s->in_flight++;
    s->stats.submitted++;
    s->cv.notify_one();
    return TBR_OK;
}

static bool bad_request(const tbr_server *s, const tbr_frame_desc *frame) {
    return !s || !frame || !frame->points2D || !frame->points3D || frame->n < 3;
}

tbr_status tbr_server_submit(tbr_server *s, const tbr_frame_desc *frame, uint64_t *request_id) {
    if (bad_request(s, frame)) return fail(TBR_ERR_INVALID_ARG, "bad frame");
    if (!(frame->K[0] > 0) || !(frame->K[1] > 0)) return fail(TBR_ERR_INVALID_ARG, "bad camera");
    auto r = std::make_unique<ServerRequest>();
    r->uv.assign(frame->points2D, frame->points2D + 2 * frame->n);
    r->xyz.assign(frame->points3D, frame->points3D + 3 * frame->n);
    return server_enqueue(s, std::move(r), frame, request_id);
}

tbr_status tbr_server_submit_nocopy(tbr_server *s, const tbr_frame_desc *frame, uint64_t *request_id) {
    if (bad_request(s, frame)) return fail(TBR_ERR_INVALID_ARG, "bad frame");
    if (!(frame->K[0] > 0) || !(frame->K[1] > 0)) return fail(TBR_ERR_INVALID_ARG, "bad camera");
    auto r = std::make_unique<ServerRequest>();
    r->ext_uv = frame->points2D;
    r->ext_xyz = frame->points3D;
    return server_enqueue(s, std::move(r), frame, request_id);
}

tbr_status tbr_server_get_stats(tbr_server *s, tbr_server_stats *out) {
    if (!s || !out) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    return TBR_OK;
}

tbr_status tbr_server_poll(tbr_server *s, tbr_server_result *out, int32_t max, int32_t *n_out) {
    if (!s || !out || max < 0) return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    const int m = std::min<int>(max, (int)s->done.size());
    for (int i = 0; i < m; ++i) out[i] = s->done[i];
    s->done.erase(s->done.begin(), s->done.begin() + m);
    if (n_out) *n_out = m;
    if (m == 0 && s->error) return fail(s->error, s->error_msg);
    return m ? TBR_OK : TBR_ERR_NOT_READY;
}

tbr_status tbr_server_cancel(tbr_server *s, uint64_t request_id) {
    if (!s) return fail(TBR_ERR_INVALID_ARG, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto &q : s->queue)
        if (q->id == request_id) {
            q->cancelled = true;
            s->cv.notify_one();
            return TBR_OK;
        }
    s->cancel_ids.push_back(request_id);
    return TBR_OK;
}

tbr_status tbr_server_drain(tbr_server *s) {
    if (!s) return fail(TBR_ERR_INVALID_ARG, "NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return s->in_flight == 0 || s->error; });
    return s->error ? fail(s->error, s->error_msg) : TBR_OK;
}

void tbr_server_destroy(tbr_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    cudaStreamSynchronize(s->E.stream);
    server_free(s);
}

tbr_status tbr_debug_score_samples(tbr_context *ctx, const double *points2D, const double *points3D,
                                   int64_t n, const double K[4], double max_reproj_error,
                                   const int32_t *triples, int64_t n_samples, int64_t *ids, double *poses,
                                   float *scores32, int64_t *counts, int64_t cap, int64_t *n_hyp,
                                   const tbr_ext_options *ext) {
    if (!ctx || !points2D || !points3D || !K || !triples || n < 3 || n_samples < 1)
        return fail(TBR_ERR_INVALID_ARG, "bad arguments");
    Engine &E = ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(ctx);
    RunOptions o;
    if (ext) {  // scoring shape only
        tbr_ext_options sh;
        std::memset(&sh, 0, sizeof(sh));
        sh.hyp_per_thread = ext->hyp_per_thread;
        sh.points_per_iter = ext->points_per_iter;
        sh.chunk_points = ext->chunk_points;
        o = make_run_options(nullptr, nullptr, &sh);
    }
    o.B = n_samples;
    o.force_samples = n_samples;
    o.skip_refine = 1;
    FrameHost fh{points2D, points3D, n, {K[0], K[1], K[2], K[3]}, 0, max_reproj_error, triples, n_samples};
    if (4 * n_samples > E.P.max_hyps) return fail(TBR_ERR_OOM, "too many samples for the hypothesis pool");
    std::vector<int> slots;
    int64_t max_n = 0;
    TBR_CUDA(cudaSetDevice(E.device));
    TBR_CUDA(cudaMemsetAsync(E.P.counters, 0, 8 * kCNum, E.stream));
    tbr_status st = admit_frames(E, {fh}, o, slots, max_n);
    if (st) return st;
    E.launch_prep(1, max_n);
    k_plan<<<1, kMaxActive, 0, E.stream>>>(E.P);
    k_sample_p3p<<<E.p3p_grid, 128, 0, E.stream>>>(E.P);
    k_score_plan<<<1, kMaxActive, 0, E.stream>>>(E.P);
    E.launch_score(E.P, o.hr, o.pp, E.stream);
    if (counts) k_debug_counts<<<E.num_sms * 4, 256, 0, E.stream>>>(E.P);
    TBR_CUDA(cudaGetLastError());
    FrameDev fd;
    TBR_CUDA(cudaMemcpyAsync(&fd, E.P.frames + slots[0], sizeof(FrameDev), cudaMemcpyDeviceToHost, E.stream));
    TBR_CUDA(cudaMemcpyAsync(E.h_counters, E.P.counters, 8 * kCNum, cudaMemcpyDeviceToHost, E.stream));
    TBR_CUDA(cudaStreamSynchronize(E.stream));
    if (E.h_counters[kCError]) {
        E.blocks.release(fd.blk_off, fd.n_blocks);
        E.free_slots.push_back(slots[0]);
        return fail(TBR_ERR_TIMEOUT, "device error flag set");
    }
    const int64_t nh = fd.hyp_count;
    std::vector<int64_t> hid(nh);
    std::vector<double> hp(12 * nh);
    std::vector<float> hs(nh);
    std::vector<int64_t> hc(nh);
    TBR_CUDA(cudaMemcpy(hid.data(), E.P.hId + fd.hyp_base, 8 * nh, cudaMemcpyDeviceToHost));
    TBR_CUDA(cudaMemcpy(hp.data(), E.P.hP64 + 12 * fd.hyp_base, 96 * nh, cudaMemcpyDeviceToHost));
    TBR_CUDA(cudaMemcpy(hs.data(), E.P.hS32 + fd.hyp_base, 4 * nh, cudaMemcpyDeviceToHost));
    if (counts) TBR_CUDA(cudaMemcpy(hc.data(), E.P.dbg_counts, 8 * nh, cudaMemcpyDeviceToHost));
    E.blocks.release(fd.blk_off, fd.n_blocks);
    E.free_slots.push_back(slots[0]);
    // Sort by id (sample order, solution order).
    std::vector<int64_t> order(nh);
    for (int64_t i = 0; i < nh; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return hid[a] < hid[b]; });
    const int64_t m = std::min(nh, cap);
    for (int64_t k = 0; k < m; ++k) {
        const int64_t i = order[k];
        if (ids) ids[k] = hid[i];
        if (poses) std::memcpy(poses + 12 * k, &hp[12 * i], 96);
        if (scores32) scores32[k] = hs[i];
        if (counts) counts[k] = hc[i];
    }
    if (n_hyp) *n_hyp = m;
    return TBR_OK;
}

}  // extern "C"

// ======================================================= no-allocation path ==
// An FP64 MSAC scorer for callers that cannot allocate device memory: code
// that runs where cudaMalloc is unavailable or forbidden -- inside another
// library's memory pool, in an allocation-free real-time loop, or under a
// host runtime that owns every device allocation. The caller passes device
// inputs and outputs; the only other memory it touches is the fixed scratch
// array below, which every GPU that loads this library holds until exit.
namespace tbr {

constexpr int kNoAllocMaxPoses = 1024;   // poses per call
constexpr int kNoAllocChunks = 32;       // point chunks per pose (partial sums)

struct NoAllocScratch {
    double part_s[kNoAllocMaxPoses][kNoAllocChunks];
    int part_c[kNoAllocMaxPoses][kNoAllocChunks];
    unsigned arrive[kNoAllocMaxPoses];   // cleared at the start of every call
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// One CTA per (pose, chunk): the per-point formula of msac.cuh:18-56, a block
// sum into the scratch partials, and the last chunk of each pose adding the
// partials in chunk order plus (n - count) * sq_thr (ransac.cuh:322).
__global__ void __launch_bounds__(256) k_msac_noalloc(NoAllocScratch *sc, const double *xn, const double *X,
                                                      int64_t n, const double *poses, double sq_thr,
                                                      double *scores, int64_t *counts) {
    __shared__ double ss[8];
    __shared__ int scnt[8];
    __shared__ unsigned prev;
    const int p = blockIdx.y, ch = blockIdx.x;
    const int64_t per = (n + kNoAllocChunks - 1) / kNoAllocChunks;
    const int64_t i0 = (int64_t)ch * per, i1 = i0 + per < n ? i0 + per : n;
    double M[12];
#pragma unroll
    for (int e = 0; e < 12; ++e) M[e] = poses[12 * p + e];
    double s = 0.0;
    int c = 0;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        const double X0 = X[3 * i], X1 = X[3 * i + 1], X2 = X[3 * i + 2];
        const double z0 = M[0] * X0 + M[1] * X1 + M[2] * X2 + M[3];
        const double z1 = M[4] * X0 + M[5] * X1 + M[6] * X2 + M[7];
        const double z2 = M[8] * X0 + M[9] * X1 + M[10] * X2 + M[11];
        const double inv_z2 = 1.0 / z2;
        const double r0 = z0 * inv_z2 - xn[2 * i], r1 = z1 * inv_z2 - xn[2 * i + 1];
        const double r_sq = r0 * r0 + r1 * r1;
        if (r_sq < sq_thr && z2 > 0.0) {
            s += r_sq;
            ++c;
        }
    }
    s = warp_sum(s);
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0) {
        ss[threadIdx.x >> 5] = s;
        scnt[threadIdx.x >> 5] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0.0;
        int C = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            S += ss[k];
            C += scnt[k];
        }
        sc->part_s[p][ch] = S;
        sc->part_c[p][ch] = C;
        __threadfence();
        prev = atomicAdd(&sc->arrive[p], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0 && prev == (unsigned)(kNoAllocChunks - 1)) {
        __threadfence();
        double S = 0.0;
        int64_t C = 0;
        for (int q = 0; q < kNoAllocChunks; ++q) {
            S += __ldcg(&sc->part_s[p][q]);
            C += __ldcg(&sc->part_c[p][q]);
        }
        scores[p] = S + (double)(n - C) * sq_thr;
        counts[p] = C;
    }
}

// Device address of the scratch array, resolved once per device.
static std::mutex g_noalloc_mu;
static std::unordered_map<int, NoAllocScratch *> g_noalloc_ptr;

}  // namespace tbr

tbr_status tbr_debug_bounded_wait(tbr_context *ctx, uint32_t polls) {
    if (!ctx || polls < 1 || polls > (1u << 22)) return fail(TBR_ERR_INVALID_ARG, "polls must be in [1, 2^22]");
    Engine &E = ctx->E;
    std::lock_guard<std::mutex> lk(E.mu);
    retire_tickets(ctx);
    TBR_CUDA(cudaSetDevice(E.device));
    TBR_CUDA(cudaMemsetAsync(E.P.counters, 0, 8 * kCNum, E.stream));
    k_debug_bounded_wait<<<1, 32, 0, E.stream>>>(E.P.counters, polls);
    TBR_CUDA(cudaGetLastError());
    TBR_CUDA(cudaMemcpyAsync(E.h_counters, E.P.counters, 8 * kCNum, cudaMemcpyDeviceToHost, E.stream));
    TBR_CUDA(cudaStreamSynchronize(E.stream));
    TBR_CUDA(cudaMemsetAsync(E.P.counters, 0, 8 * kCNum, E.stream));
    TBR_CUDA(cudaStreamSynchronize(E.stream));
    if (E.h_counters[kCError] & kErrTimeout) return fail(TBR_ERR_TIMEOUT, "bounded device wait expired");
    return TBR_OK;
}

extern "C" tbr_status tbr_msac_score_noalloc(const double *x_dev, const double *X_dev, int64_t n,
                                              const double *poses_dev, int32_t n_poses, double sq_threshold,
                                              double *scores_dev, int64_t *counts_dev, void *stream) {
    if (!x_dev || !X_dev || !poses_dev || !scores_dev || !counts_dev || n < 1 || n_poses < 0)
        return fail(TBR_ERR_INVALID_ARG, "tbr_msac_score_noalloc: bad arguments");
    if (!(sq_threshold > 0.0) || !std::isfinite(sq_threshold))
        return fail(TBR_ERR_INVALID_ARG, "tbr_msac_score_noalloc: sq_threshold must be positive and finite");
    if (n_poses > kNoAllocMaxPoses)
        return fail(TBR_ERR_INVALID_ARG, "tbr_msac_score_noalloc: at most 1024 poses per call (fixed scratch size)");
    if (n_poses == 0) return TBR_OK;
    int dev = 0;
    TBR_CUDA(cudaGetDevice(&dev));
    if (stream) {  // the scratch address is the current device's: the stream must belong to it
        int sdev = -1;
        TBR_CUDA(cudaStreamGetDevice((cudaStream_t)stream, &sdev));
        if (sdev != dev)
            return fail(TBR_ERR_INVALID_ARG,
                        "tbr_msac_score_noalloc: the stream belongs to device " + std::to_string(sdev) +
                            " but device " + std::to_string(dev) + " is current; make the stream's device current");
    }
    NoAllocScratch *sc = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        auto it = g_noalloc_ptr.find(dev);
        if (it == g_noalloc_ptr.end()) {
            // First call on this device (the device is current): translate the
            // symbol into a device address. Host code must not use the
            // symbol's own name as a pointer; it is only a host-side stand-in.
            void *ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess)
                return fail(TBR_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            it = g_noalloc_ptr.emplace(dev, (NoAllocScratch *)ptr).first;
        }
        sc = it->second;
    }
    cudaStream_t st = (cudaStream_t)stream;
    TBR_CUDA(cudaMemsetAsync(sc->arrive, 0, sizeof(unsigned) * n_poses, st));
    k_msac_noalloc<<<dim3(kNoAllocChunks, n_poses), 256, 0, st>>>(sc, x_dev, X_dev, n, poses_dev, sq_threshold,
                                                                    scores_dev, counts_dev);
    TBR_CUDA(cudaGetLastError());
    return TBR_OK;
}
