// Drop-in for <TbrCudaPnP/pose_utils.cuh>: quaternion helpers on Eigen types,
// q = (w, x, y, z), with the reference's conventions (pose_utils.cuh:13-188):
// Shepperd-branch rotation-to-quaternion with normalisation, post-multiplied
// exponential step, Taylor form of exp below 1e-6 rad.
#ifndef TBR_SHIM_POSE_UTILS_CUH
#define TBR_SHIM_POSE_UTILS_CUH

#include <cmath>

#include <Eigen/Dense>
#include <TbrCudaPnP/config.h>

namespace TbrCudaPnP {

TBR_HD inline Eigen::Matrix<double, 4, 1> rotmat_to_quat(const Eigen::Matrix<double, 3, 3> &R) {
    double w, x, y, z;
    const double tr = R(0, 0) + R(1, 1) + R(2, 2);
    if (tr > 0.0) {
        const double s = 0.5 / std::sqrt(tr + 1.0);
        w = 0.25 / s;
        x = (R(2, 1) - R(1, 2)) * s;
        y = (R(0, 2) - R(2, 0)) * s;
        z = (R(1, 0) - R(0, 1)) * s;
    } else if (R(0, 0) > R(1, 1) && R(0, 0) > R(2, 2)) {
        const double s = 2.0 * std::sqrt(1.0 + R(0, 0) - R(1, 1) - R(2, 2));
        w = (R(2, 1) - R(1, 2)) / s;
        x = 0.25 * s;
        y = (R(0, 1) + R(1, 0)) / s;
        z = (R(0, 2) + R(2, 0)) / s;
    } else if (R(1, 1) > R(2, 2)) {
        const double s = 2.0 * std::sqrt(1.0 + R(1, 1) - R(0, 0) - R(2, 2));
        w = (R(0, 2) - R(2, 0)) / s;
        x = (R(0, 1) + R(1, 0)) / s;
        y = 0.25 * s;
        z = (R(1, 2) + R(2, 1)) / s;
    } else {
        const double s = 2.0 * std::sqrt(1.0 + R(2, 2) - R(0, 0) - R(1, 1));
        w = (R(1, 0) - R(0, 1)) / s;
        x = (R(0, 2) + R(2, 0)) / s;
        y = (R(1, 2) + R(2, 1)) / s;
        z = 0.25 * s;
    }
    Eigen::Matrix<double, 4, 1> q(w, x, y, z);
    q.normalize();
    return q;
}

TBR_HD inline Eigen::Matrix<double, 3, 3> quat_to_rotmat(const Eigen::Matrix<double, 4, 1> &q) {
    const double w = q(0), x = q(1), y = q(2), z = q(3);
    Eigen::Matrix<double, 3, 3> R;
    R(0, 0) = 1.0 - 2.0 * (y * y + z * z);
    R(0, 1) = 2.0 * (x * y - z * w);
    R(0, 2) = 2.0 * (x * z + y * w);
    R(1, 0) = 2.0 * (x * y + z * w);
    R(1, 1) = 1.0 - 2.0 * (x * x + z * z);
    R(1, 2) = 2.0 * (y * z - x * w);
    R(2, 0) = 2.0 * (x * z - y * w);
    R(2, 1) = 2.0 * (y * z + x * w);
    R(2, 2) = 1.0 - 2.0 * (x * x + y * y);
    return R;
}

TBR_HD inline Eigen::Matrix<double, 4, 1> quat_multiply(const Eigen::Matrix<double, 4, 1> &a,
                                                        const Eigen::Matrix<double, 4, 1> &b) {
    return Eigen::Matrix<double, 4, 1>(a(0) * b(0) - a(1) * b(1) - a(2) * b(2) - a(3) * b(3),
                                       a(0) * b(1) + a(1) * b(0) + a(2) * b(3) - a(3) * b(2),
                                       a(0) * b(2) + a(2) * b(0) - a(1) * b(3) + a(3) * b(1),
                                       a(0) * b(3) + a(1) * b(2) - a(2) * b(1) + a(3) * b(0));
}

TBR_HD inline Eigen::Matrix<double, 4, 1> quat_conj(const Eigen::Matrix<double, 4, 1> &q) {
    return Eigen::Matrix<double, 4, 1>(q(0), -q(1), -q(2), -q(3));
}

// R(q) p via two quaternion products.
TBR_HD inline Eigen::Matrix<double, 3, 1> quat_rotate(const Eigen::Matrix<double, 4, 1> &q,
                                                      const Eigen::Matrix<double, 3, 1> &p) {
    const Eigen::Matrix<double, 4, 1> v(0.0, p(0), p(1), p(2));
    const Eigen::Matrix<double, 4, 1> r = quat_multiply(quat_multiply(q, v), quat_conj(q));
    return Eigen::Matrix<double, 3, 1>(r(1), r(2), r(3));
}

TBR_HD inline Eigen::Matrix<double, 4, 1> quat_exp(const Eigen::Matrix<double, 3, 1> &w) {
    const double th2 = w.squaredNorm(), th = std::sqrt(th2);
    double re, im;
    if (th > 1e-6) {
        re = std::cos(0.5 * th);
        im = std::sin(0.5 * th) / th;
    } else {
        re = 1.0 - th2 / 8.0 + th2 * th2 / 384.0;
        im = 0.5 - th2 / 48.0 + th2 * th2 / 3840.0;
        const double s = std::sqrt(re * re + im * im * th2);
        re /= s;
        im /= s;
    }
    return Eigen::Matrix<double, 4, 1>(re, im * w(0), im * w(1), im * w(2));
}

TBR_HD inline Eigen::Matrix<double, 4, 1> quat_step_pre(const Eigen::Matrix<double, 4, 1> &q,
                                                        const Eigen::Matrix<double, 3, 1> &w) {
    return quat_multiply(quat_exp(w), q);
}

TBR_HD inline Eigen::Matrix<double, 4, 1> quat_step_post(const Eigen::Matrix<double, 4, 1> &q,
                                                         const Eigen::Matrix<double, 3, 1> &w) {
    return quat_multiply(q, quat_exp(w));
}

}  // namespace TbrCudaPnP

#endif
