// Precision-overloaded math used by the cell models.  The double overloads
// call CUDA's double-precision functions; the float overloads call the
// single-precision ones.  MB_FAST_FP32_MATH switches the float exp/log to the
// hardware approximations (ex2.approx / lg2.approx through __expf/__logf).
#pragma once
#include <cuda_runtime.h>

// Device code compiled with and without MB_FAST_FP32_MATH lives in different
// inline namespaces, so the two translation units never share a definition.
#ifdef MB_FAST_FP32_MATH
#define MB_NS_BEGIN namespace mb { inline namespace fastf {
#else
#define MB_NS_BEGIN namespace mb { inline namespace accf {
#endif
#define MB_NS_END } }

MB_NS_BEGIN

__device__ __forceinline__ double mexp(double x) { return exp(x); }
__device__ __forceinline__ double mlog(double x) { return log(x); }
__device__ __forceinline__ double msqrt(double x) { return sqrt(x); }
__device__ __forceinline__ double mexpm1(double x) { return expm1(x); }
__device__ __forceinline__ double mpow(double x, double y) { return pow(x, y); }

#ifdef MB_FAST_FP32_MATH
__device__ __forceinline__ float mexp(float x) { return __expf(x); }
__device__ __forceinline__ float mlog(float x) { return __logf(x); }
__device__ __forceinline__ float mpow(float x, float y) { return __powf(x, y); }
#else
__device__ __forceinline__ float mpow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ float mexp(float x) { return expf(x); }
__device__ __forceinline__ float mlog(float x) { return logf(x); }
#endif
__device__ __forceinline__ float msqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ float mexpm1(float x) { return expm1f(x); }

MB_NS_END
