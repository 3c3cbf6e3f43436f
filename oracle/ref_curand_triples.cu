/*
 * The reference's minimal samples, drawn on the GPU exactly as its RANSAC
 * kernel draws them (TEST INFRASTRUCTURE, built into oracle/_ref by
 * `make -C oracle refcuda`).
 *
 * Round r (r = 0, 1, ...) seeds one cuRAND XORWOW state per sample slot b with
 * curand_init(r * B + 1234, b, 0) (turbo_ransac.cu:159-160 with
 * ransac_utils.cuh:14-19: the seed is the running sample count plus 1234, the
 * subsequence the block index). Thread 0 of the slot then draws three
 * uniforms, maps each to floor(u * n) clamped to n - 1, and redraws all three
 * until they are distinct (ransac.cuh:176-196). The triples are written in
 * sample order r * B + b, so replaying them through the engine or the FP64
 * oracle scores the reference's own minimal sets. cuRAND is called, not
 * reimplemented.
 *
 * The redraw loop is bounded here (2^20 attempts, far beyond any n >= 3);
 * a slot that gives up is reported through the return value.
 */
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <cstdint>

namespace {

__global__ void k_reference_triples(int64_t n, int64_t B, int32_t *out, int *failed) {
    const int64_t b = blockIdx.x, r = blockIdx.y;
    if (threadIdx.x != 0 || b >= B) return;
    curandState st;
    curand_init((unsigned long long)(r * B + 1234), (unsigned long long)b, 0ull, &st);
    int s[3] = {0, 1, 2};
    bool valid = false;
    for (int attempt = 0; attempt < (1 << 20) && !valid; ++attempt) {
        for (int i = 0; i < 3; ++i) {
            const float u = curand_uniform(&st);
            s[i] = static_cast<int>(u * n);
            if (s[i] >= n) s[i] = (int)(n - 1);
        }
        valid = (s[0] != s[1] && s[0] != s[2] && s[1] != s[2]);
    }
    if (!valid) atomicExch(failed, 1);
    int32_t *o = out + 3 * (r * B + b);
    o[0] = s[0];
    o[1] = s[1];
    o[2] = s[2];
}

}  // namespace

extern "C" {

/* out: host array of rounds * B * 3 int32. Returns 0 on success, 1 if a slot
 * found no distinct triple, 2 on a CUDA error or bad arguments. */
int ref_curand_triples(int64_t n, int64_t B, int32_t rounds, int32_t *out) {
    if (n < 3 || B < 1 || B > 0x7fffffff || rounds < 1 || rounds > 65535 || !out) return 2;
    const size_t bytes = sizeof(int32_t) * 3 * (size_t)B * (size_t)rounds;
    int32_t *d_out = nullptr;
    int *d_failed = nullptr;
    if (cudaMalloc(&d_out, bytes) != cudaSuccess) return 2;
    if (cudaMalloc(&d_failed, sizeof(int)) != cudaSuccess) {
        cudaFree(d_out);
        return 2;
    }
    int failed = 0;
    cudaMemset(d_failed, 0, sizeof(int));
    k_reference_triples<<<dim3((unsigned)B, (unsigned)rounds), 32>>>(n, B, d_out, d_failed);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(out, d_out, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&failed, d_failed, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d_out);
    cudaFree(d_failed);
    if (e != cudaSuccess) return 2;
    return failed ? 1 : 0;
}

}
