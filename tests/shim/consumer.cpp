// A caller of the TbrCudaPnP C++ API written the way the reference's evaluator
// calls it (TbrMain/src/main.cu:160-202): reads one frame from a binary file
// (n, K[4], then n*(u, v, X, Y, Z) doubles), calls estimate_absolute_pose_cuda
// and prints the pose as one line: "ok q0 q1 q2 q3 t0 t1 t2 num_inliers".
// Built against include/ (the drop-in headers) and linked with libtbr.so.
#include <TbrCudaPnP/header.h>

#include <cstdio>
#include <fstream>
#include <vector>

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    std::ifstream in(argv[1], std::ios::binary);
    int64_t n = 0;
    in.read((char *)&n, 8);
    std::vector<double> K(4);
    in.read((char *)K.data(), 32);
    std::vector<Eigen::Vector2d> p2d;
    std::vector<Eigen::Vector3d> p3d;
    for (int64_t i = 0; i < n; ++i) {
        double r[5];
        in.read((char *)r, 40);
        p2d.emplace_back(r[0], r[1]);
        p3d.emplace_back(r[2], r[3], r[4]);
    }
    TbrCudaPnP::Camera_cuda cam;
    cam.width = static_cast<int>(K[2]) * 2;
    cam.height = static_cast<int>(K[3]) * 2;
    cam.params = K.data();
    TbrCudaPnP::RansacOptions_cuda ropt;
    ropt.max_iterations = 1000;
    ropt.success_prob = 0.9999;
    ropt.max_reproj_error = 4.0;
    if (argc > 2) ropt.seed = std::strtoull(argv[2], nullptr, 10);
    TbrCudaPnP::BundleOptions_cuda bopt;
    TbrCudaPnP::CameraPose_cuda pose;
    std::vector<char> inl(p2d.size(), 0);
    TbrCudaPnP::RansacStats_cuda st = TbrCudaPnP::estimate_absolute_pose_cuda(p2d, p3d, cam, ropt, bopt, &pose, &inl);
    Eigen::Matrix4d T = pose.Rt_homo();
    std::printf("%s %.17g %.17g %.17g %.17g %.17g %.17g %.17g %zu %g\n", st.num_inliers ? "ok" : "fail", pose.q(0),
                pose.q(1), pose.q(2), pose.q(3), T(0, 3), T(1, 3), T(2, 3), st.num_inliers, st.model_score);
    return 0;
}
