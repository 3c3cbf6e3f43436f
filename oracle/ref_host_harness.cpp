// Host harness over the reference's OWN source (TEST INFRASTRUCTURE).
//
// Built by oracle/Makefile from the reference tree into oracle/_ref/ (never
// committed). It compiles the reference's header code -- p3p.cuh,
// p3p_utils.cuh, pose_utils.cuh, msac.cuh, robust_loss.cuh, lm_utils.cuh,
// jaco.cuh, lm.cuh -- with g++ through the stubs in oracle/refshim and the
// Eigen subset in oracle/eigen_subset, and links the reference's entry.cu
// unchanged. Two GPU-only pieces are replaced by harness glue:
//  * turbo_ransac_pnp (turbo_ransac.cu) returns a pose the caller injects,
//    so entry.cu's post-RANSAC orchestration runs from the reference source;
//  * bundle_adjust_cuda (ba.cu:31-108 is cudaMalloc/copy glue) runs the
//    reference's lm_impl<CameraJacobianAccumulator_cuda> as one host thread.
// The exported ref_* functions give known answers for the oracle's tests.
#include <cuda_runtime.h>
#include <Eigen/Dense>
#include <cstdint>
#include <cstring>
#include <vector>

#include <TbrCudaPnP/p3p.cuh>
#include <TbrCudaPnP/msac.cuh>
#include <TbrCudaPnP/pose.cuh>
#include <TbrCudaPnP/camera.cuh>
#include <TbrCudaPnP/utils.h>
#include <TbrCudaPnP/lm.cuh>
#include <TbrCudaPnP/jaco.cuh>
#include <TbrCudaPnP/lm_utils.cuh>
#include <TbrCudaPnP/robust_loss.cuh>
#include <TbrCudaPnP/entry.h>
#include <TbrCudaPnP/turbo_ransac.cuh>
#include <TbrCudaPnP/ba.cuh>

using namespace TbrCudaPnP;

static Eigen::Matrix<double, 4, 4> g_injected_pose = Eigen::Matrix<double, 4, 4>::Identity();

namespace TbrCudaPnP {
void turbo_ransac_pnp(const int, const Eigen::Matrix<double, 2, 1> *, const Eigen::Matrix<double, 3, 1> *,
                      const RansacOptions_cuda &, RansacStats_cuda &, Eigen::Matrix<double, 4, 4> &result_pose,
                      int *) {
    result_pose = g_injected_pose;
}

BundleStats_cuda bundle_adjust_cuda(const int points_num, const Eigen::Matrix<double, 2, 1> *x,
                                    const Eigen::Matrix<double, 3, 1> *X, const Camera_cuda &camera,
                                    CameraPose_cuda *pose, const int, const BundleOptions_cuda &opt,
                                    const double *) {
    CameraJacobianAccumulator_cuda accum;
    accum.x = reinterpret_cast<const double *>(x);
    accum.X = reinterpret_cast<const double *>(X);
    accum.cam_k = camera.params;
    accum.n = points_num;
    CameraJacobianAccumulator_cuda::param_t p;
    p.q = pose[0].q;
    p.t = pose[0].t;
    lm_impl<decltype(accum)>(accum, &p, opt);
    *pose = p;
    return BundleStats_cuda();
}
}  // namespace TbrCudaPnP

extern "C" {

int ref_p3p(const double *x, const double *X, double *out) {
    Eigen::Matrix<double, 3, 1> xs[3], Xs[3];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) { xs[i](k) = x[3 * i + k]; Xs[i](k) = X[3 * i + k]; }
    Eigen::Matrix<double, 4, 4> sols[4];
    int n = p3p<double>(xs, Xs, sols);
    for (int s = 0; s < n; ++s)
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) out[12 * s + 4 * r + c] = sols[s](r, c);
    return n;
}

void ref_bearing(double x, double y, double out[3]) {
    Eigen::Matrix<double, 3, 1> v;
    v(0) = x; v(1) = y; v(2) = 1;
    v.normalize();
    for (int k = 0; k < 3; ++k) out[k] = v(k);
}

void ref_msac(const double *xn, const double *X, int64_t n, const double *P, double sq_thr,
              double *score, int64_t *count) {
    Eigen::Matrix<double, 4, 4> pose = Eigen::Matrix<double, 4, 4>::Identity();
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) pose(r, c) = P[4 * r + c];
    double s = 0.0;
    int64_t cnt = 0;
    for (int64_t i = 0; i < n; ++i) {
        SharedPointData pt;
        pt.p2d(0) = xn[2 * i]; pt.p2d(1) = xn[2 * i + 1];
        pt.p3d(0) = X[3 * i]; pt.p3d(1) = X[3 * i + 1]; pt.p3d(2) = X[3 * i + 2];
        pt.is_inlier = 0; pt.point_score = 0.0;
        compute_msac_scores(sq_thr, pose, pt);
        s += pt.point_score;
        cnt += pt.is_inlier;
    }
    *score = s + (n - cnt) * sq_thr;
    *count = cnt;
}

void ref_rotmat_to_quat(const double *R, double q[4]) {
    Eigen::Matrix<double, 3, 3> M;
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) M(r, c) = R[3 * r + c];
    Eigen::Matrix<double, 4, 1> v = rotmat_to_quat(M);
    for (int k = 0; k < 4; ++k) q[k] = v(k);
}

void ref_quat_to_rotmat(const double q[4], double *R) {
    Eigen::Matrix<double, 4, 1> v(q[0], q[1], q[2], q[3]);
    Eigen::Matrix<double, 3, 3> M = quat_to_rotmat(v);
    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) R[3 * r + c] = M(r, c);
}

void ref_quat_step_post(const double q[4], const double w[3], double out[4]) {
    Eigen::Matrix<double, 4, 1> v(q[0], q[1], q[2], q[3]);
    Eigen::Matrix<double, 3, 1> d(w[0], w[1], w[2]);
    Eigen::Matrix<double, 4, 1> r = quat_step_post(v, d);
    for (int k = 0; k < 4; ++k) out[k] = r(k);
}

void ref_solve_cholesky6(const double *A, const double *b, double *x) {
    Eigen::Matrix<double, 6, 6> M;
    Eigen::Matrix<double, 6, 1> v, s;
    for (int r = 0; r < 6; ++r) { v(r) = b[r]; for (int c = 0; c < 6; ++c) M(r, c) = A[6 * r + c]; }
    solve_cholesky<double, 6>(M, v, s);
    for (int r = 0; r < 6; ++r) x[r] = s(r);
}

double ref_cauchy_loss(double scale, double r2) { return CauchyLoss_cuda(scale).loss(r2); }
double ref_cauchy_weight(double scale, double r2) { return CauchyLoss_cuda(scale).weight(r2); }

// lm_impl on (x, X) with camera (fx, fy, cx, cy): q, t refined in place.
void ref_lm(const double *x, const double *X, int64_t n, const double cam[4], double q[4], double t[3],
            int64_t max_iterations, double loss_scale) {
    std::vector<Eigen::Matrix<double, 2, 1>> xs(n);
    std::vector<Eigen::Matrix<double, 3, 1>> Xs(n);
    for (int64_t i = 0; i < n; ++i) {
        xs[i](0) = x[2 * i]; xs[i](1) = x[2 * i + 1];
        Xs[i](0) = X[3 * i]; Xs[i](1) = X[3 * i + 1]; Xs[i](2) = X[3 * i + 2];
    }
    double k[4] = {cam[0], cam[1], cam[2], cam[3]};
    Camera_cuda c;
    c.params = k;
    CameraPose_cuda p(Eigen::Matrix<double, 4, 1>(q[0], q[1], q[2], q[3]),
                      Eigen::Matrix<double, 3, 1>(t[0], t[1], t[2]));
    BundleOptions_cuda opt;
    opt.max_iterations = (size_t)max_iterations;
    opt.loss_scale = loss_scale;
    bundle_adjust_cuda((int)n, xs.data(), Xs.data(), c, &p, 1, opt);
    for (int i = 0; i < 4; ++i) q[i] = p.q(i);
    for (int i = 0; i < 3; ++i) t[i] = p.t(i);
}

// entry.cu's estimate_absolute_pose_cuda with the RANSAC pose injected
// (P: 3x4 row-major). inliers: n bytes.
void ref_estimate_from_pose(const double *uv, const double *X, int64_t n, const double K[4],
                            double max_reproj_error, const double *P, double q[4], double t[3],
                            uint8_t *inliers) {
    g_injected_pose.setIdentity();
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) g_injected_pose(r, c) = P[4 * r + c];
    std::vector<Eigen::Vector2d> p2(n);
    std::vector<Eigen::Vector3d> p3(n);
    for (int64_t i = 0; i < n; ++i) {
        p2[i](0) = uv[2 * i]; p2[i](1) = uv[2 * i + 1];
        p3[i](0) = X[3 * i]; p3[i](1) = X[3 * i + 1]; p3[i](2) = X[3 * i + 2];
    }
    std::vector<double> params = {K[0], K[1], K[2], K[3]};
    Camera_cuda cam;
    cam.width = 640;
    cam.height = 480;
    cam.params = params.data();
    RansacOptions_cuda ropt;
    ropt.max_reproj_error = max_reproj_error;
    BundleOptions_cuda bopt;
    CameraPose_cuda pose;
    std::vector<char> inl;
    estimate_absolute_pose_cuda(p2, p3, cam, ropt, bopt, &pose, &inl);
    for (int i = 0; i < 4; ++i) q[i] = pose.q(i);
    for (int i = 0; i < 3; ++i) t[i] = pose.t(i);
    for (int64_t i = 0; i < n; ++i) inliers[i] = (uint8_t)inl[i];
}

}  // extern "C"
