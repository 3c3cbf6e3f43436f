// Drop-in for <TbrCudaPnP/ba.cuh> (ba.cuh:17-24): LM refinement over libtbr.so.
// As in the reference (ba.cu:121-129 with jaco.cuh:36,123) the loss is Cauchy
// with opt.loss_scale and the weights do not enter the cost.
#ifndef TBR_SHIM_BA_CUH
#define TBR_SHIM_BA_CUH

#include <TbrCudaPnP/entry.h>

namespace TbrCudaPnP {

inline BundleStats_cuda bundle_adjust_cuda(const int points_num, const Eigen::Matrix<double, 2, 1> *x,
                                           const Eigen::Matrix<double, 3, 1> *X, const Camera_cuda &camera,
                                           CameraPose_cuda *pose, const int poses_num, const BundleOptions_cuda &opt,
                                           const double *weights = nullptr) {
    (void)poses_num;
    BundleStats_cuda bs{};
    std::vector<double> xs(2 * (size_t)points_num), Xs(3 * (size_t)points_num);
    for (int k = 0; k < points_num; ++k) {
        xs[2 * k] = x[k](0);
        xs[2 * k + 1] = x[k](1);
        Xs[3 * k] = X[k](0);
        Xs[3 * k + 1] = X[k](1);
        Xs[3 * k + 2] = X[k](2);
    }
    const double K[4] = {camera.params[0], camera.params[1], camera.params[2], camera.params[3]};
    double q[4] = {pose->q(0), pose->q(1), pose->q(2), pose->q(3)};
    double t[3] = {pose->t(0), pose->t(1), pose->t(2)};
    const tbr_bundle_options bo = detail::to_c(opt);
    tbr_stats st;
    tbr_context *ctx = detail::default_context();
    if (!ctx || tbr_bundle_adjust(ctx, xs.data(), Xs.data(), points_num, K, q, t, &bo, weights, nullptr, &st) != TBR_OK) {
        std::fprintf(stderr, "TbrCudaPnP::bundle_adjust_cuda: %s\n", tbr_last_error());
        return bs;
    }
    pose->q = Eigen::Matrix<double, 4, 1>(q[0], q[1], q[2], q[3]);
    pose->t = Eigen::Matrix<double, 3, 1>(t[0], t[1], t[2]);
    bs.iterations = (size_t)st.lm_iterations;
    bs.initial_cost = st.lm_initial_cost;
    bs.cost = st.lm_cost;
    bs.invalid_steps = (size_t)st.lm_invalid_steps;
    return bs;
}

}  // namespace TbrCudaPnP

#endif
