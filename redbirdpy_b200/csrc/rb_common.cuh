// Shared helpers of the redbird_b200 CUDA library: status/error plumbing,
// real/complex scalar arithmetic and warp reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <cstdarg>
#include <string>

#include "../../include/redbird_b200.h"

namespace rb {

// thread-local message returned by rb_last_error()
std::string& last_error();
int fail(int code, const char* fmt, ...);

#define RB_CUDA_TRY(call)                                                        \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess)                                                       \
      return ::rb::fail(RB_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,      \
                        cudaGetErrorString(e_));                                 \
  } while (0)

#define RB_LAUNCH_CHECK() RB_CUDA_TRY(cudaGetLastError())

#define RB_TRY(expr)                 \
  do {                               \
    int s_ = (expr);                 \
    if (s_ != RB_OK) return s_;      \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int kWarp = 32;
constexpr double kC0 = 299792458000.0;  // speed of light, mm/s

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// ------------------------------------------------------------------ scalars
typedef float2 cfloat;
typedef double2 cdouble;

template <typename T> struct Scalar;
template <> struct Scalar<float> {
  typedef float real;
  typedef double acc;  // dot-product accumulator
  static constexpr bool is_complex = false;
};
template <> struct Scalar<double> {
  typedef double real;
  typedef double acc;
  static constexpr bool is_complex = false;
};
template <> struct Scalar<cfloat> {
  typedef float real;
  typedef cdouble acc;
  static constexpr bool is_complex = true;
};
template <> struct Scalar<cdouble> {
  typedef double real;
  typedef cdouble acc;
  static constexpr bool is_complex = true;
};

__host__ __device__ __forceinline__ float s_zero(float) { return 0.f; }
__host__ __device__ __forceinline__ double s_zero(double) { return 0.0; }
__host__ __device__ __forceinline__ cfloat s_zero(cfloat) { return make_float2(0.f, 0.f); }
__host__ __device__ __forceinline__ cdouble s_zero(cdouble) { return make_double2(0.0, 0.0); }

// a*b + c (complex: full complex product, no conjugation)
__device__ __forceinline__ float s_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double s_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ cfloat s_fma(cfloat a, cfloat b, cfloat c) {
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}
__device__ __forceinline__ cdouble s_fma(cdouble a, cdouble b, cdouble c) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ float s_mul(float a, float b) { return a * b; }
__device__ __forceinline__ double s_mul(double a, double b) { return a * b; }
__device__ __forceinline__ cfloat s_mul(cfloat a, cfloat b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ cdouble s_mul(cdouble a, cdouble b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float s_add(float a, float b) { return a + b; }
__device__ __forceinline__ double s_add(double a, double b) { return a + b; }
__device__ __forceinline__ cfloat s_add(cfloat a, cfloat b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cdouble s_add(cdouble a, cdouble b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float s_sub(float a, float b) { return a - b; }
__device__ __forceinline__ double s_sub(double a, double b) { return a - b; }
__device__ __forceinline__ cfloat s_sub(cfloat a, cfloat b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cdouble s_sub(cdouble a, cdouble b) { return make_double2(a.x - b.x, a.y - b.y); }
// |a|^2 in double
__device__ __forceinline__ double s_abs2(float a) { return (double)a * a; }
__device__ __forceinline__ double s_abs2(double a) { return a * a; }
__device__ __forceinline__ double s_abs2(cfloat a) { return (double)a.x * a.x + (double)a.y * a.y; }
__device__ __forceinline__ double s_abs2(cdouble a) { return a.x * a.x + a.y * a.y; }

// widening / narrowing conversions
__device__ __forceinline__ double to_acc(float a) { return a; }
__device__ __forceinline__ double to_acc(double a) { return a; }
__device__ __forceinline__ cdouble to_acc(cfloat a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ cdouble to_acc(cdouble a) { return a; }
template <typename T> __device__ __forceinline__ T from_acc(double a);
template <> __device__ __forceinline__ float from_acc<float>(double a) { return (float)a; }
template <> __device__ __forceinline__ double from_acc<double>(double a) { return a; }
template <typename T> __device__ __forceinline__ T from_cacc(cdouble a);
template <> __device__ __forceinline__ cfloat from_cacc<cfloat>(cdouble a) {
  return make_float2((float)a.x, (float)a.y);
}
template <> __device__ __forceinline__ cdouble from_cacc<cdouble>(cdouble a) { return a; }

__device__ __forceinline__ double acc_fma(float a, float b, double c) { return fma((double)a, (double)b, c); }
__device__ __forceinline__ double acc_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ cdouble acc_fma(cfloat a, cfloat b, cdouble c) {
  return s_fma(to_acc(a), to_acc(b), c);
}
__device__ __forceinline__ cdouble acc_fma(cdouble a, cdouble b, cdouble c) { return s_fma(a, b, c); }

// -------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// exclusive scan helper (int32) used by the setup kernels; n+1 outputs
size_t scan_work_bytes(int64_t n);
int scan_exclusive(const int32_t* in, int32_t* out, int64_t n, void* work, size_t work_bytes,
                   cudaStream_t st);

}  // namespace rb
