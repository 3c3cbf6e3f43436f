// Drop-in for <TbrCudaPnP/entry.h> (entry.h:13-25): estimate_absolute_pose_cuda
// and get_inliers_mx with the reference's signatures, implemented inline over
// the C ABI of libtbr.so (link with -ltbr). Differences from the reference:
// CUDA failures are reported on stderr and returned as stats with
// num_inliers = 0 and the identity pose instead of exit() (cudaCheck.h:4-14);
// RansacStats_cuda carries the real sample and inlier counts (the reference
// returns it unfilled, entry.cu:69,141) while model_score stays 0 as there.
#ifndef TBR_SHIM_ENTRY_H
#define TBR_SHIM_ENTRY_H

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

#include <tbr.h>
#include <TbrCudaPnP/camera.cuh>
#include <TbrCudaPnP/pose.cuh>
#include <TbrCudaPnP/utils.h>

namespace TbrCudaPnP {
namespace detail {

// One context per process, created on first use on device TBR_DEVICE (default 0).
inline tbr_context *default_context() {
    static tbr_context *ctx = [] {
        tbr_context *c = nullptr;
        const char *d = std::getenv("TBR_DEVICE");
        if (tbr_context_create(d ? std::atoi(d) : 0, 0, &c) != TBR_OK) {
            std::fprintf(stderr, "TbrCudaPnP: %s\n", tbr_last_error());
            return (tbr_context *)nullptr;
        }
        return c;
    }();
    return ctx;
}

inline tbr_ransac_options to_c(const RansacOptions_cuda &o) {
    tbr_ransac_options r;
    r.max_iterations = o.max_iterations;
    r.min_iterations = o.min_iterations;
    r.dyn_num_trials_mult = o.dyn_num_trials_mult;
    r.success_prob = o.success_prob;
    r.max_reproj_error = o.max_reproj_error;
    r.max_epipolar_error = o.max_epipolar_error;
    r.seed = o.seed;
    r.progressive_sampling = o.progressive_sampling;
    r.max_prosac_iterations = o.max_prosac_iterations;
    r.real_focal_check = o.real_focal_check;
    r.score_initial_model = o.score_initial_model;
    return r;
}

inline tbr_bundle_options to_c(const BundleOptions_cuda &o) {
    tbr_bundle_options b;
    b.max_iterations = o.max_iterations;
    b.loss_type = (int32_t)o.loss_type;
    b.loss_scale = o.loss_scale;
    b.gradient_tol = o.gradient_tol;
    b.step_tol = o.step_tol;
    b.initial_lambda = o.initial_lambda;
    b.min_lambda = o.min_lambda;
    b.max_lambda = o.max_lambda;
    b.verbose = o.verbose;
    return b;
}

}  // namespace detail

inline void get_inliers_mx(const CameraPose_cuda &pose, const std::vector<Eigen::Vector2d> &x,
                           const std::vector<Eigen::Vector3d> &X, double sq_threshold, std::vector<char> *inliers) {
    const size_t n = x.size();
    inliers->assign(n, 0);
    if (n == 0) return;
    std::vector<double> xs(2 * n), Xs(3 * n);
    for (size_t k = 0; k < n; ++k) {
        xs[2 * k] = x[k](0);
        xs[2 * k + 1] = x[k](1);
        Xs[3 * k] = X[k](0);
        Xs[3 * k + 1] = X[k](1);
        Xs[3 * k + 2] = X[k](2);
    }
    const double q[4] = {pose.q(0), pose.q(1), pose.q(2), pose.q(3)};
    const double t[3] = {pose.t(0), pose.t(1), pose.t(2)};
    std::vector<uint8_t> m(n);
    tbr_context *ctx = detail::default_context();
    if (!ctx || tbr_get_inliers(ctx, q, t, xs.data(), Xs.data(), (int64_t)n, sq_threshold, m.data(), nullptr) != TBR_OK) {
        std::fprintf(stderr, "TbrCudaPnP::get_inliers_mx: %s\n", tbr_last_error());
        return;
    }
    for (size_t k = 0; k < n; ++k) (*inliers)[k] = (char)m[k];
}

inline RansacStats_cuda estimate_absolute_pose_cuda(const std::vector<Eigen::Vector2d> &points2D,
                                                    const std::vector<Eigen::Vector3d> &points3D,
                                                    const Camera_cuda &camera, const RansacOptions_cuda &ransac_opt,
                                                    const BundleOptions_cuda &bundle_opt, CameraPose_cuda *pose,
                                                    std::vector<char> *inliers) {
    RansacStats_cuda stats;
    const size_t n = points2D.size();
    *pose = CameraPose_cuda();
    if (inliers) inliers->assign(n, 0);
    if (points3D.size() != n) {
        std::fprintf(stderr, "TbrCudaPnP: 2D and 3D point counts must match\n");
        stats.num_inliers = 0;
        return stats;
    }
    std::vector<double> uv(2 * n), X(3 * n);
    for (size_t k = 0; k < n; ++k) {
        uv[2 * k] = points2D[k](0);
        uv[2 * k + 1] = points2D[k](1);
        X[3 * k] = points3D[k](0);
        X[3 * k + 1] = points3D[k](1);
        X[3 * k + 2] = points3D[k](2);
    }
    const double K[4] = {camera.params[0], camera.params[1], camera.params[2], camera.params[3]};
    const tbr_ransac_options ro = detail::to_c(ransac_opt);
    const tbr_bundle_options bo = detail::to_c(bundle_opt);
    double q[4], t[3];
    std::vector<uint8_t> m(n);
    tbr_stats st;
    tbr_context *ctx = detail::default_context();
    if (!ctx || tbr_estimate_absolute_pose(ctx, uv.data(), X.data(), (int64_t)n, K, camera.width, camera.height, &ro,
                                           &bo, nullptr, q, t, m.data(), &st) != TBR_OK) {
        std::fprintf(stderr, "TbrCudaPnP::estimate_absolute_pose_cuda: %s\n", tbr_last_error());
        stats.num_inliers = 0;
        return stats;
    }
    pose->q = Eigen::Matrix<double, 4, 1>(q[0], q[1], q[2], q[3]);
    pose->t = Eigen::Matrix<double, 3, 1>(t[0], t[1], t[2]);
    if (inliers)
        for (size_t k = 0; k < n; ++k) (*inliers)[k] = (char)m[k];
    stats.iterations = (size_t)st.samples;
    stats.num_inliers = (size_t)st.num_inliers;
    stats.inlier_ratio = st.inlier_ratio;
    stats.refinements = 1;
    stats.model_score = 0;  // entry.cu:141
    return stats;
}

}  // namespace TbrCudaPnP

#endif
