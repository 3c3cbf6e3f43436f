/*
 * The reference's RANSAC kernel launched directly, for a scoring-bound timing
 * (measurement infrastructure for the comparison arm, built into oracle/_ref by
 * `make -C oracle refcuda`).
 *
 * The reference cannot switch its early stop off, so its whole call cannot
 * score an exact sample count; this harness reproduces the launch sequence of
 * one round of turbo_ransac_pnp (turbo_ransac.cu:78-97 for the shared-memory
 * and tile sizing, :159-174 for the two launches) with B blocks -- B minimal
 * samples, each P3P'd and scored in FP64 over all n points by one block -- and
 * times the scoring kernel with CUDA events. Inputs must be valid frames with
 * n >= 3 (the reference's sampler loops until it draws distinct indices).
 */
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <TbrCudaPnP/ransac.cuh>

#include <cfloat>
#include <cstdint>
#include <vector>

extern "C" {

/* x_norm: n*2 normalized image points, X: n*3. Runs `reps` rounds of B samples
 * (the first round's samples, i.e. the reference's seed 1234). Returns 0 on
 * success; *ms = mean device ms of one turbo_ransac_pnp_kernel launch,
 * *best = lowest block score of the last launch. */
int ref_scoring_kernel(const double *x_norm, const double *X, int n, int B, double max_sq_error, int reps,
                       float *ms, double *best) {
    using namespace TbrCudaPnP;
    if (n < 3 || B < 1 || reps < 1 || !x_norm || !X || !ms || !best) return 2;
    double *d_x = nullptr, *d_X = nullptr, *d_pose = nullptr, *d_score = nullptr;
    int *d_inl = nullptr;
    curandState *d_rand = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = 0;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == 0) rc = 3;
        return rc == 0;
    };
    ok(cudaMalloc(&d_x, sizeof(double) * 2 * n));
    ok(cudaMalloc(&d_X, sizeof(double) * 3 * n));
    ok(cudaMalloc(&d_pose, sizeof(double) * 16 * B));
    ok(cudaMalloc(&d_score, sizeof(double) * B));
    ok(cudaMalloc(&d_inl, sizeof(int) * B));
    ok(cudaMalloc(&d_rand, sizeof(curandState) * B));
    ok(cudaEventCreate(&e0));
    ok(cudaEventCreate(&e1));
    if (rc == 0) {
        ok(cudaMemcpy(d_x, x_norm, sizeof(double) * 2 * n, cudaMemcpyHostToDevice));
        ok(cudaMemcpy(d_X, X, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
        int device = 0, max_shared = 0;
        ok(cudaGetDevice(&device));
        ok(cudaDeviceGetAttribute(&max_shared, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        const int shared_mem_size = max_shared > 65536 ? 65536 : max_shared;
        ok(cudaFuncSetAttribute(turbo_ransac_pnp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                shared_mem_size));
        int tile_size = shared_mem_size / (int)sizeof(SharedPointData);
        tile_size = tile_size > 384 ? 384 : tile_size;
        float total = 0.f;
        for (int r = 0; r < reps && rc == 0; ++r) {
            setup_rand_kernel<<<B, tile_size>>>(d_rand, 1234UL);
            ok(cudaGetLastError());
            ok(cudaEventRecord(e0));
            turbo_ransac_pnp_kernel<<<B, tile_size, shared_mem_size>>>(d_rand, tile_size, n, d_x, d_X, d_pose,
                                                                       max_sq_error, d_score, d_inl);
            ok(cudaGetLastError());
            ok(cudaEventRecord(e1));
            ok(cudaEventSynchronize(e1));
            float t = 0.f;
            ok(cudaEventElapsedTime(&t, e0, e1));
            total += t;
        }
        if (rc == 0) {
            std::vector<double> s(B);
            ok(cudaMemcpy(s.data(), d_score, sizeof(double) * B, cudaMemcpyDeviceToHost));
            double m = DBL_MAX;
            for (double v : s) m = v < m ? v : m;
            *best = m;
            *ms = total / reps;
        }
    }
    cudaFree(d_x);
    cudaFree(d_X);
    cudaFree(d_pose);
    cudaFree(d_score);
    cudaFree(d_inl);
    cudaFree(d_rand);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return rc;
}

}
