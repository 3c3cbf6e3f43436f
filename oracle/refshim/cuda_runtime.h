// Host-compilation stub for <cuda_runtime.h> (TEST INFRASTRUCTURE).
// Lets the reference's device headers compile with g++ as single-thread host
// code: CUDA qualifiers vanish, __shared__ becomes function-static, and the
// "block" is one thread, so warp shuffles contribute nothing and block-wide
// reductions reduce to the thread's own sequential sum.
#ifndef TBR_REFSHIM_CUDA_RUNTIME_H
#define TBR_REFSHIM_CUDA_RUNTIME_H
#include <algorithm>
#include <cassert>
#include <cfloat>
#include <cmath>
#include <cstdio>
#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
#define __shared__ static
#define __align__(n) alignas(n)
struct tbr_refshim_dim3 { unsigned x, y, z; };
static const tbr_refshim_dim3 threadIdx = {0u, 0u, 0u};
static const tbr_refshim_dim3 blockIdx = {0u, 0u, 0u};
static const tbr_refshim_dim3 blockDim = {1u, 1u, 1u};
static const int warpSize = 32;
template <class T> inline T __shfl_down_sync(unsigned, T, int) { return T(0); }
inline void __syncthreads() {}
#endif
