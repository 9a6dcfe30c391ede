// Shared helpers for the sinc-DVR orbital-RHS CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#define SINCGPU_OK 0
#define SINCGPU_EINVAL 1
#define SINCGPU_ECUDA 2
#define SINCGPU_ENOMEM 3
#define SINCGPU_ESTATE 4
#define SINCGPU_ETIMEOUT 5
#define SINCGPU_ERANGE 6

namespace sincgpu {

// Records the message of the last failure for sincgpu_last_error().
void set_error(const char* fmt, ...);

#define SG_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      ::sincgpu::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call,                 \
                           cudaGetErrorString(e_));                                    \
      return SINCGPU_ECUDA;                                                            \
    }                                                                                  \
  } while (0)

#define SG_CHECK(cond, code, ...)                                                      \
  do {                                                                                 \
    if (!(cond)) {                                                                     \
      ::sincgpu::set_error(__VA_ARGS__);                                               \
      return (code);                                                                   \
    }                                                                                  \
  } while (0)

#define SG_TRY(expr)                                                                   \
  do {                                                                                 \
    int r_ = (expr);                                                                   \
    if (r_ != SINCGPU_OK) return r_;                                                   \
  } while (0)

// Counts kernel launches of this library (sincgpu_launch_count).
void count_launch();

// Kernel launch check: catches configuration errors right after launch.
#define SG_LAUNCHED()            \
  do {                           \
    ::sincgpu::count_launch();   \
    SG_CUDA(cudaGetLastError()); \
  } while (0)

__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
#ifdef __CUDACC__
// acc += v*m with explicit FMAs (one rounding order wherever it is used)
__device__ __forceinline__ void cfma(double2& acc, double2 v, double2 m) {
  acc.x = fma(v.x, m.x, fma(-v.y, m.y, acc.x));
  acc.y = fma(v.x, m.y, fma(v.y, m.x, acc.y));
}
#endif
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a*conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) {
  return make_double2(a.x * s, a.y * s);
}

// single-precision complex helpers (precision form of the Coulomb passes)
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// real type and constructor of a complex type
template <class C>
struct CplxTraits;
template <>
struct CplxTraits<double2> {
  using Real = double;
  __host__ __device__ static double2 make(double re, double im) { return make_double2(re, im); }
};
template <>
struct CplxTraits<float2> {
  using Real = float;
  __host__ __device__ static float2 make(double re, double im) { return make_float2((float)re, (float)im); }
};
template <class C>
__host__ __device__ __forceinline__ C cvt(double2 v) {
  return CplxTraits<C>::make(v.x, v.y);
}
__host__ __device__ __forceinline__ double2 widen(double2 v) { return v; }
__host__ __device__ __forceinline__ double2 widen(float2 v) { return make_double2(v.x, v.y); }

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace sincgpu
