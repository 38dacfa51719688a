// Vector load/store helpers for AoS records (2 or 4 values of T per element).
// Internal to libop2b.
#pragma once

#include <cuda_runtime.h>

namespace op2b {


template <typename T> struct Vec;
template <> struct Vec<double> {
  static __device__ __forceinline__ void ld2(const double *p, double &a, double &b) {
    double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    a = v.x;
    b = v.y;
  }
  static __device__ __forceinline__ void ld4(const double *p, double *o) {
    double2 v0 = __ldg(reinterpret_cast<const double2 *>(p));
    double2 v1 = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    o[0] = v0.x; o[1] = v0.y; o[2] = v1.x; o[3] = v1.y;
  }
  static __device__ __forceinline__ void ld4_rw(const double *p, double *o) {
    double2 v0 = reinterpret_cast<const double2 *>(p)[0];
    double2 v1 = reinterpret_cast<const double2 *>(p)[1];
    o[0] = v0.x; o[1] = v0.y; o[2] = v1.x; o[3] = v1.y;
  }
  static __device__ __forceinline__ void st4(double *p, const double *v) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
  }
  // streaming (evict-first) forms for data touched once per launch
  static __device__ __forceinline__ void ld4_cs(const double *p, double *o) {
    double2 v0 = __ldcs(reinterpret_cast<const double2 *>(p));
    double2 v1 = __ldcs(reinterpret_cast<const double2 *>(p) + 1);
    o[0] = v0.x; o[1] = v0.y; o[2] = v1.x; o[3] = v1.y;
  }
  static __device__ __forceinline__ void st4_cs(double *p, const double *v) {
    __stcs(reinterpret_cast<double2 *>(p), make_double2(v[0], v[1]));
    __stcs(reinterpret_cast<double2 *>(p) + 1, make_double2(v[2], v[3]));
  }
  // shared-memory records (16-byte aligned)
  static __device__ __forceinline__ void st4_shared(double *p, const double *v) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
  }
  static __device__ __forceinline__ void ld4_shared(const double *p, double *o) {
    const double2 v0 = reinterpret_cast<const double2 *>(p)[0];
    const double2 v1 = reinterpret_cast<const double2 *>(p)[1];
    o[0] = v0.x; o[1] = v0.y; o[2] = v1.x; o[3] = v1.y;
  }
};
template <> struct Vec<float> {
  static __device__ __forceinline__ void ld2(const float *p, float &a, float &b) {
    float2 v = __ldg(reinterpret_cast<const float2 *>(p));
    a = v.x;
    b = v.y;
  }
  static __device__ __forceinline__ void ld4(const float *p, float *o) {
    float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
  static __device__ __forceinline__ void ld4_rw(const float *p, float *o) {
    float4 v = *reinterpret_cast<const float4 *>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
  static __device__ __forceinline__ void st4(float *p, const float *v) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
  static __device__ __forceinline__ void ld4_cs(const float *p, float *o) {
    float4 v = __ldcs(reinterpret_cast<const float4 *>(p));
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
  static __device__ __forceinline__ void st4_cs(float *p, const float *v) {
    __stcs(reinterpret_cast<float4 *>(p), make_float4(v[0], v[1], v[2], v[3]));
  }
  static __device__ __forceinline__ void st4_shared(float *p, const float *v) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  }
  static __device__ __forceinline__ void ld4_shared(const float *p, float *o) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
  }
};

}  // namespace op2b
