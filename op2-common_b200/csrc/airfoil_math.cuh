// Per-element Airfoil arithmetic shared by every device loop variant.
//
// The expression trees are those of the reference kernels
// (apps/c/airfoil/airfoil_plain/dp/adt_calc.h:1-27, res_calc.h:1-33,
// bres_calc.h:1-35, update.h:1-19), including the float-literal promotions
// (1.0f, 0.5f), because the plain FP64 path is required to reproduce the
// reference's values: this file is compiled with --fmad=false, so every
// double operation is rounded once exactly as the reference's sequential
// build does with -ffp-contract=off.  T = double for the plain path and
// T = float for the mixed-precision form's flux loops.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace op2b {

template <typename T> struct AirConst {
  T gam, gm1, cfl, eps;
  T qinf[4];
};

template <typename T> __device__ __forceinline__ T dsqrt(T v);
template <> __device__ __forceinline__ double dsqrt<double>(double v) { return sqrt(v); }
template <> __device__ __forceinline__ float dsqrt<float>(float v) { return sqrtf(v); }
template <typename T> __device__ __forceinline__ T dabs(T v);
template <> __device__ __forceinline__ double dabs<double>(double v) { return fabs(v); }
template <> __device__ __forceinline__ float dabs<float>(float v) { return fabsf(v); }

// adt_calc.h:1-27 -- local time step of a cell from its 4 nodes and q.
template <typename T>
__device__ __forceinline__ T air_adt(T x1x, T x1y, T x2x, T x2y, T x3x, T x3y,
                                     T x4x, T x4y, T q0, T q1, T q2, T q3,
                                     const AirConst<T> &k) {
  T dx, dy, ri, u, v, c, adt;
  ri = (T)1.0f / q0;
  u = ri * q1;
  v = ri * q2;
  c = dsqrt<T>(k.gam * k.gm1 * (ri * q3 - (T)0.5f * (u * u + v * v)));
  dx = x2x - x1x;
  dy = x2y - x1y;
  adt = dabs<T>(u * dy - v * dx) + c * dsqrt<T>(dx * dx + dy * dy);
  dx = x3x - x2x;
  dy = x3y - x2y;
  adt += dabs<T>(u * dy - v * dx) + c * dsqrt<T>(dx * dx + dy * dy);
  dx = x4x - x3x;
  dy = x4y - x3y;
  adt += dabs<T>(u * dy - v * dx) + c * dsqrt<T>(dx * dx + dy * dy);
  dx = x1x - x4x;
  dy = x1y - x4y;
  adt += dabs<T>(u * dy - v * dx) + c * dsqrt<T>(dx * dx + dy * dy);
  return adt / k.cfl;
}

// res_calc.h:1-33 -- flux f[4] across an interior edge; the caller adds f
// to cell 1 and subtracts it from cell 2.
template <typename T>
__device__ __forceinline__ void air_flux(T x1x, T x1y, T x2x, T x2y,
                                         const T *q1, const T *q2, T adt1,
                                         T adt2, const AirConst<T> &k, T *f) {
  T dx, dy, mu, ri, p1, vol1, p2, vol2;
  dx = x1x - x2x;
  dy = x1y - x2y;
  ri = (T)1.0f / q1[0];
  p1 = k.gm1 * (q1[3] - (T)0.5f * ri * (q1[1] * q1[1] + q1[2] * q1[2]));
  vol1 = ri * (q1[1] * dy - q1[2] * dx);
  ri = (T)1.0f / q2[0];
  p2 = k.gm1 * (q2[3] - (T)0.5f * ri * (q2[1] * q2[1] + q2[2] * q2[2]));
  vol2 = ri * (q2[1] * dy - q2[2] * dx);
  mu = (T)0.5f * (adt1 + adt2) * k.eps;
  f[0] = (T)0.5f * (vol1 * q1[0] + vol2 * q2[0]) + mu * (q1[0] - q2[0]);
  f[1] = (T)0.5f * (vol1 * q1[1] + p1 * dy + vol2 * q2[1] + p2 * dy) +
         mu * (q1[1] - q2[1]);
  f[2] = (T)0.5f * (vol1 * q1[2] - p1 * dx + vol2 * q2[2] - p2 * dx) +
         mu * (q1[2] - q2[2]);
  f[3] = (T)0.5f * (vol1 * (q1[3] + p1) + vol2 * (q2[3] + p2)) +
         mu * (q1[3] - q2[3]);
}

// The per-cell terms of res_calc.h:8-13 -- ri = 1/q[0] and the pressure p --
// which depend on the cell alone.  air_flux_prim is air_flux with them passed
// in: the same operations in the same order, so a cell that owns several
// edges computes its own terms once and gets bit-identical fluxes.
template <typename T>
__device__ __forceinline__ void air_prim(const T *q, const AirConst<T> &k, T &ri, T &p) {
  ri = (T)1.0f / q[0];
  p = k.gm1 * (q[3] - (T)0.5f * ri * (q[1] * q[1] + q[2] * q[2]));
}

template <typename T>
__device__ __forceinline__ void air_flux_prim(T x1x, T x1y, T x2x, T x2y, const T *q1,
                                              const T *q2, T ri1, T p1, T ri2, T p2, T adt1,
                                              T adt2, const AirConst<T> &k, T *f) {
  T dx, dy, mu, vol1, vol2;
  dx = x1x - x2x;
  dy = x1y - x2y;
  vol1 = ri1 * (q1[1] * dy - q1[2] * dx);
  vol2 = ri2 * (q2[1] * dy - q2[2] * dx);
  mu = (T)0.5f * (adt1 + adt2) * k.eps;
  f[0] = (T)0.5f * (vol1 * q1[0] + vol2 * q2[0]) + mu * (q1[0] - q2[0]);
  f[1] = (T)0.5f * (vol1 * q1[1] + p1 * dy + vol2 * q2[1] + p2 * dy) +
         mu * (q1[1] - q2[1]);
  f[2] = (T)0.5f * (vol1 * q1[2] - p1 * dx + vol2 * q2[2] - p2 * dx) +
         mu * (q1[2] - q2[2]);
  f[3] = (T)0.5f * (vol1 * (q1[3] + p1) + vol2 * (q2[3] + p2)) +
         mu * (q1[3] - q2[3]);
}

// bres_calc.h:1-35 -- increment r[4] of the cell on a boundary edge
// (wall: pressure only, r[0] = r[3] = 0; far field: flux against qinf).
template <typename T>
__device__ __forceinline__ void air_bflux(T x1x, T x1y, T x2x, T x2y,
                                          const T *q1, T adt1, int bound,
                                          const AirConst<T> &k, T *r) {
  T dx, dy, mu, ri, p1, vol1, p2, vol2;
  dx = x1x - x2x;
  dy = x1y - x2y;
  ri = (T)1.0f / q1[0];
  p1 = k.gm1 * (q1[3] - (T)0.5f * ri * (q1[1] * q1[1] + q1[2] * q1[2]));
  if (bound == 1) {
    r[0] = (T)0;
    r[1] = +p1 * dy;
    r[2] = -p1 * dx;
    r[3] = (T)0;
  } else {
    const T *qi = k.qinf;
    vol1 = ri * (q1[1] * dy - q1[2] * dx);
    ri = (T)1.0f / qi[0];
    p2 = k.gm1 * (qi[3] - (T)0.5f * ri * (qi[1] * qi[1] + qi[2] * qi[2]));
    vol2 = ri * (qi[1] * dy - qi[2] * dx);
    mu = adt1 * k.eps;
    r[0] = (T)0.5f * (vol1 * q1[0] + vol2 * qi[0]) + mu * (q1[0] - qi[0]);
    r[1] = (T)0.5f * (vol1 * q1[1] + p1 * dy + vol2 * qi[1] + p2 * dy) +
           mu * (q1[1] - qi[1]);
    r[2] = (T)0.5f * (vol1 * q1[2] - p1 * dx + vol2 * qi[2] - p2 * dx) +
           mu * (q1[2] - qi[2]);
    r[3] = (T)0.5f * (vol1 * (q1[3] + p1) + vol2 * (qi[3] + p2)) +
           mu * (q1[3] - qi[3]);
  }
}

// air_bflux with the cell's own terms ri = 1/q1[0] and p1 (air_prim) passed
// in: the same operations in the same order, so the values are bit-identical.
template <typename T>
__device__ __forceinline__ void air_bflux_prim(T x1x, T x1y, T x2x, T x2y, const T *q1, T ri1,
                                               T p1, T adt1, int bound, const AirConst<T> &k,
                                               T *r) {
  T dx, dy, mu, ri, p2, vol1, vol2;
  dx = x1x - x2x;
  dy = x1y - x2y;
  if (bound == 1) {
    r[0] = (T)0;
    r[1] = +p1 * dy;
    r[2] = -p1 * dx;
    r[3] = (T)0;
  } else {
    const T *qi = k.qinf;
    vol1 = ri1 * (q1[1] * dy - q1[2] * dx);
    ri = (T)1.0f / qi[0];
    p2 = k.gm1 * (qi[3] - (T)0.5f * ri * (qi[1] * qi[1] + qi[2] * qi[2]));
    vol2 = ri * (qi[1] * dy - qi[2] * dx);
    mu = adt1 * k.eps;
    r[0] = (T)0.5f * (vol1 * q1[0] + vol2 * qi[0]) + mu * (q1[0] - qi[0]);
    r[1] = (T)0.5f * (vol1 * q1[1] + p1 * dy + vol2 * qi[1] + p2 * dy) +
           mu * (q1[1] - qi[1]);
    r[2] = (T)0.5f * (vol1 * q1[2] - p1 * dx + vol2 * qi[2] - p2 * dx) +
           mu * (q1[2] - qi[2]);
    r[3] = (T)0.5f * (vol1 * (q1[3] + p1) + vol2 * (qi[3] + p2)) +
           mu * (q1[3] - qi[3]);
  }
}

} // namespace op2b
