// airfoil_math.cuh -- the airfoil user kernels as device functions, and the
// vector loads and stores the loop kernels share (airfoil.cu, group.cu).
//
// The user-kernel arithmetic (airfoil/*.h) is restated term for term in the
// reference's evaluation order; the library is compiled with -fmad=false and
// IEEE division and square root, so every per-element value is
// bit-identical to the reference's x86 build.
#pragma once

#include <cuda_runtime.h>

namespace op2b {

// ---------------------------------------------------------- vector I/O ----
__device__ __forceinline__ void ld2(const float *p, float v[2]) {
  float2 t = __ldg(reinterpret_cast<const float2 *>(p));
  v[0] = t.x; v[1] = t.y;
}
__device__ __forceinline__ void ld2(const double *p, double v[2]) {
  double2 t = __ldg(reinterpret_cast<const double2 *>(p));
  v[0] = t.x; v[1] = t.y;
}
__device__ __forceinline__ void ld4(const float *p, float v[4]) {
  float4 t = __ldg(reinterpret_cast<const float4 *>(p));
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ld4(const double *p, double v[4]) {
  double2 a = __ldg(reinterpret_cast<const double2 *>(p));
  double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
// plain (coherent) loads for data the kernel also writes
__device__ __forceinline__ void ldw4(const float *p, float v[4]) {
  float4 t = *reinterpret_cast<const float4 *>(p);
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
__device__ __forceinline__ void ldw4(const double *p, double v[4]) {
  double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void st4(float *p, const float v[4]) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double *p, const double v[4]) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}

// 1/x rounded to nearest: IEEE division of one by x, i.e. the reference's
// `1.0f/x` on x86, bit for bit, in fewer instructions than a general divide
__device__ __forceinline__ float rcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }


template <class T>
struct AirConsts {
  T gam, gm1, cfl, eps, qinf[4];
};

// --------------------------------------------------------- user kernels ---
// airfoil/adt_calc.h:1-26
template <class T>
__device__ __forceinline__ T adt_calc(const T x1[2], const T x2[2], const T x3[2], const T x4[2],
                                      const T q[4], const AirConsts<T> &K) {
  T dx, dy, ri, u, v, c, adt;
  ri = rcp(q[0]);
  u = ri * q[1];
  v = ri * q[2];
  c = sqrt(K.gam * K.gm1 * (ri * q[3] - T(0.5f) * (u * u + v * v)));
  dx = x2[0] - x1[0];
  dy = x2[1] - x1[1];
  adt = fabs(u * dy - v * dx) + c * sqrt(dx * dx + dy * dy);
  dx = x3[0] - x2[0];
  dy = x3[1] - x2[1];
  adt += fabs(u * dy - v * dx) + c * sqrt(dx * dx + dy * dy);
  dx = x4[0] - x3[0];
  dy = x4[1] - x3[1];
  adt += fabs(u * dy - v * dx) + c * sqrt(dx * dx + dy * dy);
  dx = x1[0] - x4[0];
  dy = x1[1] - x4[1];
  adt += fabs(u * dy - v * dx) + c * sqrt(dx * dx + dy * dy);
  return adt / K.cfl;
}

// airfoil/res_calc.h:1-30; f is the flux added to res1 and taken from res2
template <class T>
__device__ __forceinline__ void res_flux(const T x1[2], const T x2[2], const T q1[4],
                                         const T q2[4], T adt1, T adt2, T gm1, T eps, T f[4]) {
  T dx = x1[0] - x2[0];
  T dy = x1[1] - x2[1];
  T ri = rcp(q1[0]);
  T p1 = gm1 * (q1[3] - T(0.5f) * ri * (q1[1] * q1[1] + q1[2] * q1[2]));
  T vol1 = ri * (q1[1] * dy - q1[2] * dx);
  ri = rcp(q2[0]);
  T p2 = gm1 * (q2[3] - T(0.5f) * ri * (q2[1] * q2[1] + q2[2] * q2[2]));
  T vol2 = ri * (q2[1] * dy - q2[2] * dx);
  T mu = T(0.5f) * (adt1 + adt2) * eps;
  f[0] = T(0.5f) * (vol1 * q1[0] + vol2 * q2[0]) + mu * (q1[0] - q2[0]);
  f[1] = T(0.5f) * (vol1 * q1[1] + p1 * dy + vol2 * q2[1] + p2 * dy) + mu * (q1[1] - q2[1]);
  f[2] = T(0.5f) * (vol1 * q1[2] - p1 * dx + vol2 * q2[2] - p2 * dx) + mu * (q1[2] - q2[2]);
  f[3] = T(0.5f) * (vol1 * (q1[3] + p1) + vol2 * (q2[3] + p2)) + mu * (q1[3] - q2[3]);
}

// airfoil/bres_calc.h:1-33, applied to the running value r of res1
template <class T>
__device__ __forceinline__ void bres_apply(const T x1[2], const T x2[2], const T q1[4], T adt1,
                                           int bound, const AirConsts<T> &K, T r[4]) {
  T dx = x1[0] - x2[0];
  T dy = x1[1] - x2[1];
  T ri = rcp(q1[0]);
  T p1 = K.gm1 * (q1[3] - T(0.5f) * ri * (q1[1] * q1[1] + q1[2] * q1[2]));
  if (bound == 1) {
    r[1] += +p1 * dy;
    r[2] += -p1 * dx;
  } else {
    const T *qinf = K.qinf;
    T vol1 = ri * (q1[1] * dy - q1[2] * dx);
    ri = rcp(qinf[0]);
    T p2 = K.gm1 * (qinf[3] - T(0.5f) * ri * (qinf[1] * qinf[1] + qinf[2] * qinf[2]));
    T vol2 = ri * (qinf[1] * dy - qinf[2] * dx);
    T mu = adt1 * K.eps;
    T f;
    f = T(0.5f) * (vol1 * q1[0] + vol2 * qinf[0]) + mu * (q1[0] - qinf[0]);
    r[0] += f;
    f = T(0.5f) * (vol1 * q1[1] + p1 * dy + vol2 * qinf[1] + p2 * dy) + mu * (q1[1] - qinf[1]);
    r[1] += f;
    f = T(0.5f) * (vol1 * q1[2] - p1 * dx + vol2 * qinf[2] - p2 * dx) + mu * (q1[2] - qinf[2]);
    r[2] += f;
    f = T(0.5f) * (vol1 * (q1[3] + p1) + vol2 * (qinf[3] + p2)) + mu * (q1[3] - qinf[3]);
    r[3] += f;
  }
}

// one boundary edge's increment of its cell: bres_apply onto -0.0 gives the
// exact values bres_calc adds (-0.0 where it adds nothing)
template <class T>
__device__ __forceinline__ void bres_contrib(const T x1[2], const T x2[2], const T q1[4], T adt1,
                                             int bound, const AirConsts<T> &K, T v[4]) {
  v[0] = v[1] = v[2] = v[3] = T(-0.0);
  bres_apply(x1, x2, q1, adt1, bound, K, v);
}

// the first min(W, 4) entries of cell c's list; -1 past the end
__device__ __forceinline__ void list_head(const int *__restrict__ ell, int W, int c, int k[4]) {
  if ((W & 3) == 0) {
    const int4 kk = __ldg(reinterpret_cast<const int4 *>(ell + (size_t)c * W));
    k[0] = kk.x; k[1] = kk.y; k[2] = kk.z; k[3] = kk.w;
  } else {
#pragma unroll
    for (int j = 0; j < 4; j++) k[j] = j < W ? __ldg(ell + (size_t)c * W + j) : -1;
  }
}

template <class T>
__device__ __forceinline__ void add_listed(T r[4], int k, const T f[4]) {
  if (k < 0) return;
  if (k & 1) {
    r[0] -= f[0]; r[1] -= f[1]; r[2] -= f[2]; r[3] -= f[3];
  } else {
    r[0] += f[0]; r[1] += f[1]; r[2] += f[2]; r[3] += f[3];
  }
}

}  // namespace op2b
