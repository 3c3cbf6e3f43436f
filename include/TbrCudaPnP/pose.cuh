// Drop-in for <TbrCudaPnP/pose.cuh> (pose.cuh:12-80): CameraPose_cuda with
// q = (w, x, y, z) and t, X_cam = R X + t.
#ifndef TBR_SHIM_POSE_CUH
#define TBR_SHIM_POSE_CUH

#include <TbrCudaPnP/pose_utils.cuh>

namespace TbrCudaPnP {

struct CameraPose_cuda {
    Eigen::Matrix<double, 4, 1> q;
    Eigen::Matrix<double, 3, 1> t;

    TBR_HD CameraPose_cuda() : q(1.0, 0.0, 0.0, 0.0), t(0.0, 0.0, 0.0) {}
    TBR_HD CameraPose_cuda(const Eigen::Matrix<double, 4, 1> &qq, const Eigen::Matrix<double, 3, 1> &tt)
        : q(qq), t(tt) {}
    TBR_HD CameraPose_cuda(const Eigen::Matrix<double, 3, 3> &R, const Eigen::Matrix<double, 3, 1> &tt)
        : q(rotmat_to_quat(R)), t(tt) {}

    TBR_HD Eigen::Matrix<double, 3, 3> R() const { return quat_to_rotmat(q); }
    TBR_HD Eigen::Matrix<double, 3, 4> Rt() const {
        Eigen::Matrix<double, 3, 4> m;
        const Eigen::Matrix<double, 3, 3> r = R();
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) m(i, j) = r(i, j);
            m(i, 3) = t(i);
        }
        return m;
    }
    TBR_HD Eigen::Matrix<double, 4, 4> Rt_homo() const {
        Eigen::Matrix<double, 4, 4> m = Eigen::Matrix<double, 4, 4>::Identity();
        const Eigen::Matrix<double, 3, 4> rt = Rt();
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 4; ++j) m(i, j) = rt(i, j);
        return m;
    }
    TBR_HD Eigen::Matrix<double, 3, 1> rotate(const Eigen::Matrix<double, 3, 1> &p) const { return quat_rotate(q, p); }
    TBR_HD Eigen::Matrix<double, 3, 1> derotate(const Eigen::Matrix<double, 3, 1> &p) const {
        return quat_rotate(quat_conj(q), p);
    }
    TBR_HD Eigen::Matrix<double, 3, 1> apply(const Eigen::Matrix<double, 3, 1> &p) const { return rotate(p) + t; }
    TBR_HD Eigen::Matrix<double, 3, 1> center() const { return -derotate(t); }
};

}  // namespace TbrCudaPnP

#endif
