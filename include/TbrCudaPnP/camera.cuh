// Drop-in for <TbrCudaPnP/camera.cuh> (camera.cuh:10-85): the pinhole camera
// {model_id, width, height, params = fx, fy, cx, cy} with focal() = (fx+fy)/2.
#ifndef TBR_SHIM_CAMERA_CUH
#define TBR_SHIM_CAMERA_CUH

#include <Eigen/Dense>
#include <TbrCudaPnP/config.h>

namespace TbrCudaPnP {

class Camera_cuda {
   public:
    int model_id;
    int width;
    int height;
    double *params;  // caller-owned: fx, fy, cx, cy

    TBR_HD Camera_cuda() : model_id(1), width(-1), height(-1), params(nullptr) {}

    TBR_HD void project(const Eigen::Matrix<double, 2, 1> &x, Eigen::Matrix<double, 2, 1> *xp) const {
        (*xp)(0) = params[0] * x(0) + params[2];
        (*xp)(1) = params[1] * x(1) + params[3];
    }
    TBR_HD void project_with_jac(const Eigen::Matrix<double, 2, 1> &x, Eigen::Matrix<double, 2, 1> *xp,
                                 Eigen::Matrix<double, 2, 2> *jac) const {
        project(x, xp);
        (*jac)(0, 0) = params[0];
        (*jac)(0, 1) = 0.0;
        (*jac)(1, 0) = 0.0;
        (*jac)(1, 1) = params[1];
    }
    TBR_HD void unproject(const Eigen::Matrix<double, 2, 1> &xp, Eigen::Matrix<double, 2, 1> *x) const {
        (*x)(0) = (xp(0) - params[2]) / params[0];
        (*x)(1) = (xp(1) - params[3]) / params[1];
    }
    TBR_HD double focal() const { return 0.5 * (params[0] + params[1]); }
    TBR_HD double focal_x() const { return params[0]; }
    TBR_HD double focal_y() const { return params[1]; }
    TBR_HD Eigen::Matrix<double, 2, 1> principal_point() const {
        return Eigen::Matrix<double, 2, 1>(params[2], params[3]);
    }
    void rescale(double s) {
        for (int k = 0; k < 4; ++k) params[k] *= s;
    }
};

}  // namespace TbrCudaPnP

#endif
