// Drop-in for <TbrCudaPnP/utils.h> (utils.h:14-72): the option and statistics
// structs, field for field with the reference's defaults, so callers that set
// them by name compile unchanged. libtbr.so receives them as tbr_*_options.
#ifndef TBR_SHIM_UTILS_H
#define TBR_SHIM_UTILS_H

#include <cfloat>
#include <cstddef>
#include <iostream>

#include <TbrCudaPnP/config.h>

namespace TbrCudaPnP {

struct RansacOptions_cuda {
    size_t max_iterations = 100000;  // samples per round
    size_t min_iterations = 1000;
    double dyn_num_trials_mult = 3.0;
    double success_prob = 0.9999;
    double max_reproj_error = 12.0;
    double max_epipolar_error = 1.0;
    unsigned long seed = 0;
    bool progressive_sampling = false;
    size_t max_prosac_iterations = 100000;
    bool real_focal_check = false;
    bool score_initial_model = false;
};

struct RansacStats_cuda {
    size_t refinements = 0;
    size_t iterations = 0;
    size_t num_inliers = 0;
    double inlier_ratio = 0;
    double model_score = DBL_MAX;
};

struct BundleOptions_cuda {
    size_t max_iterations = 100;
    enum LossType { TRIVIAL, TRUNCATED, HUBER, CAUCHY, TRUNCATED_LE_ZACH } loss_type = LossType::CAUCHY;
    double loss_scale = 1.0;
    double gradient_tol = 1e-10;
    double step_tol = 1e-8;
    double initial_lambda = 1e-3;
    double min_lambda = 1e-10;
    double max_lambda = 1e10;
    bool verbose = false;
};

struct BundleStats_cuda {
    size_t iterations = 0;
    double initial_cost;
    double cost;
    double lambda;
    size_t invalid_steps;
    double step_norm;
    double grad_norm;
};

}  // namespace TbrCudaPnP

#endif
