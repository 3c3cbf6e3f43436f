/*
 * Timing driver for the reference's own CUDA build (measurement infrastructure:
 * the comparison arm, not part of the product).
 *
 * Linked with the reference's unmodified sources (Module/TbrCudaPnP/src/
 * entry.cu, turbo_ransac.cu, ba.cu) by `make -C oracle refcuda`; the binary
 * lands in oracle/_ref/. It calls TbrCudaPnP::estimate_absolute_pose_cuda
 * (entry.cu:28-144) once per frame, the way TbrMain/src/main.cu:241-259 does,
 * and times each whole call on the host clock, like main.cu:185-190. The
 * reference prints to stdout inside every call (turbo_ransac.cu:200-250,
 * ba.cu:88); the caller redirects stdout, so this program writes its results
 * to a file only.
 *
 * Usage: tbr_refcuda <frames.bin> <out.bin> <warmup_calls> <max_iterations> <reproj_px>
 *
 * frames.bin: int64 n_frames, then per frame: int64 n, double K[4] (fx, fy,
 *   cx, cy), int32 width, int32 height, double uv[n*2], double xyz[n*3].
 * out.bin: per frame: double q[4], double t[3], double ms, int64 num_inliers.
 *
 * The reference's sampler loops until it draws three distinct indices and its
 * best-of-round read indexes the round's minimum; both need n >= 3 and at least
 * one P3P solution in the first round, so frames with n < 3 are refused here.
 */
#include <TbrCudaPnP/entry.h>

#include <pthread.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace {

struct Frame {
    int64_t n;
    double K[4];
    int32_t w, h;
    std::vector<Eigen::Vector2d> uv;
    std::vector<Eigen::Vector3d> xyz;
};

struct Job {
    std::vector<Frame> frames;
    int warmup;
    int max_iterations;
    double reproj_px;
    std::vector<double> out;  // 9 doubles per frame (q, t, ms, inliers as double bits)
    int rc;
};

bool read_frames(const char *path, std::vector<Frame> &frames) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    int64_t count = 0;
    bool ok = std::fread(&count, sizeof(count), 1, f) == 1 && count >= 0;
    for (int64_t i = 0; ok && i < count; ++i) {
        Frame fr;
        ok = std::fread(&fr.n, sizeof(fr.n), 1, f) == 1 && std::fread(fr.K, sizeof(double), 4, f) == 4 &&
             std::fread(&fr.w, sizeof(fr.w), 1, f) == 1 && std::fread(&fr.h, sizeof(fr.h), 1, f) == 1 &&
             fr.n >= 3;
        if (!ok) break;
        std::vector<double> uv(2 * fr.n), xyz(3 * fr.n);
        ok = std::fread(uv.data(), sizeof(double), uv.size(), f) == uv.size() &&
             std::fread(xyz.data(), sizeof(double), xyz.size(), f) == xyz.size();
        fr.uv.resize(fr.n);
        fr.xyz.resize(fr.n);
        for (int64_t k = 0; k < fr.n; ++k) {
            fr.uv[k] = Eigen::Vector2d(uv[2 * k], uv[2 * k + 1]);
            fr.xyz[k] = Eigen::Vector3d(xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]);
        }
        frames.push_back(std::move(fr));
    }
    std::fclose(f);
    return ok;
}

TbrCudaPnP::RansacStats_cuda call(const Frame &fr, const Job &job, TbrCudaPnP::CameraPose_cuda &pose,
                                  std::vector<char> &inliers) {
    TbrCudaPnP::Camera_cuda cam;
    double params[4] = {fr.K[0], fr.K[1], fr.K[2], fr.K[3]};
    cam.model_id = 1;
    cam.width = fr.w;
    cam.height = fr.h;
    cam.params = params;
    TbrCudaPnP::RansacOptions_cuda ro;
    ro.max_iterations = job.max_iterations;
    ro.max_reproj_error = job.reproj_px;
    TbrCudaPnP::BundleOptions_cuda bo;
    return TbrCudaPnP::estimate_absolute_pose_cuda(fr.uv, fr.xyz, cam, ro, bo, &pose, &inliers);
}

// The reference keeps five per-point arrays on the stack (entry.cu:51-53,
// :78-79), so the calls run on a thread with a large stack.
void *worker(void *arg) {
    Job &job = *static_cast<Job *>(arg);
    const size_t nf = job.frames.size();
    job.out.assign(nf * 9, 0.0);
    for (int w = 0; w < job.warmup && nf > 0; ++w) {
        TbrCudaPnP::CameraPose_cuda pose;
        std::vector<char> inl;
        call(job.frames[w % nf], job, pose, inl);
    }
    for (size_t i = 0; i < nf; ++i) {
        TbrCudaPnP::CameraPose_cuda pose;
        std::vector<char> inl;
        const auto t0 = std::chrono::steady_clock::now();
        call(job.frames[i], job, pose, inl);
        const auto t1 = std::chrono::steady_clock::now();
        double *o = &job.out[i * 9];
        for (int k = 0; k < 4; ++k) o[k] = pose.q(k);
        for (int k = 0; k < 3; ++k) o[4 + k] = pose.t(k);
        o[7] = std::chrono::duration<double, std::milli>(t1 - t0).count();
        int64_t cnt = 0;
        for (char c : inl) cnt += c ? 1 : 0;
        o[8] = (double)cnt;
    }
    job.rc = 0;
    return nullptr;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s frames.bin out.bin warmup max_iterations reproj_px\n", argv[0]);
        return 2;
    }
    Job job;
    job.warmup = std::atoi(argv[3]);
    job.max_iterations = std::atoi(argv[4]);
    job.reproj_px = std::atof(argv[5]);
    job.rc = 1;
    if (!read_frames(argv[1], job.frames) || job.max_iterations <= 0) {
        std::fprintf(stderr, "bad input\n");
        return 2;
    }
    pthread_attr_t attr;
    pthread_attr_init(&attr);
    pthread_attr_setstacksize(&attr, (size_t)1 << 30);
    pthread_t th;
    if (pthread_create(&th, &attr, worker, &job) != 0) return 3;
    pthread_join(th, nullptr);
    if (job.rc != 0) return job.rc;
    FILE *f = std::fopen(argv[2], "wb");
    if (!f) return 4;
    for (size_t i = 0; i < job.frames.size(); ++i) {
        const double *o = &job.out[i * 9];
        const int64_t cnt = (int64_t)o[8];
        std::fwrite(o, sizeof(double), 8, f);
        std::fwrite(&cnt, sizeof(cnt), 1, f);
    }
    std::fclose(f);
    return 0;
}
