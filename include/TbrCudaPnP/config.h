// Drop-in for the reference's <TbrCudaPnP/config.h> (Module/TbrCudaPnP/include/
// TbrCudaPnP/config.h:1-30): the precision switch and the P3P eps constants.
// As in the reference, USE_FLOAT only selects the eps constants; libtbr.so's
// P3P runs in FP64 with these float-valued thresholds.
#ifndef TBR_SHIM_CONFIG_H
#define TBR_SHIM_CONFIG_H

#if !defined(USE_FLOAT) && !defined(USE_DOUBLE)
#define USE_FLOAT
#endif

#ifdef USE_FLOAT
typedef float real_t_base;
#else
typedef double real_t_base;
#endif

namespace TbrCudaPnP {
using real_t = real_t_base;
#ifdef USE_FLOAT
constexpr real_t eps_refine_lambda = 1e-6f;
constexpr real_t eps_root2real = 1e-6f;
#else
constexpr real_t eps_refine_lambda = 1e-10;
constexpr real_t eps_root2real = 1e-12;
#endif
}  // namespace TbrCudaPnP

#if defined(__CUDACC__)
#define TBR_HD __host__ __device__
#else
#define TBR_HD
#endif

#endif
