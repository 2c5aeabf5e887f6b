// Device-side physics of the Swirl-C compressible RHS, shared by the fused
// stage kernel and the unit-level kernels.
//
// Each function states the reference lines it follows (paths relative to the
// swirl_c project root). Arithmetic runs in T (float or double).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// 1: single-precision WENO runs the neg/pos pair as f32x2 instructions
// (measured slower on B200: operand-pair moves outweigh the halved FP32
// issue count, so the scalar form is the default).
#ifndef SWC_PACKED_WENO
#define SWC_PACKED_WENO 0
#endif

namespace swc {

// physics/constant.py:17-41. Python doubles rounded once to T, as TF does
// when it mixes a Python float with a float32 tensor.
template <typename T>
struct K {
  static constexpr double kGamma = 1.4;
  static constexpr double kR = 8.314 / 0.029;
  static constexpr double kCv = kR / (kGamma - 1.0);
  static constexpr double kCp = kCv + kR;
  static constexpr double kG = 9.81;
  __device__ static constexpr T gamma() { return T(kGamma); }
  __device__ static constexpr T gm1() { return T(kGamma - 1.0); }
  __device__ static constexpr T r_gas() { return T(kR); }
  __device__ static constexpr T cp() { return T(kCp); }
  __device__ static constexpr T grav() { return T(kG); }
};

template <typename T>
__device__ __forceinline__ T dnn(T x, T y) {  // tf.math.divide_no_nan
  return y == T(0) ? T(0) : x / y;
}
// Single precision is built with -use_fast_math: 1/x is the hardware
// reciprocal approximation (<= 1 ulp) and x/y the 2-ulp division.
__device__ __forceinline__ float rcp_(float x) { return 1.0f / x; }
__device__ __forceinline__ double rcp_(double x) { return 1.0 / x; }
__device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
__device__ __forceinline__ float min_(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double min_(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float max_(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double max_(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float abs_(float a) { return fabsf(a); }
// Products that must not be contracted into an FMA: the conserved states of
// the two sides of a face, so that U_R - U_L is exactly 0 for equal states.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double abs_(double a) { return fabs(a); }

// Primitive state at a face or a cell: rho, (u, v, w), e, p, h.
template <typename T>
struct Prim {
  T r;
  T u[3];
  T e, p, h;
};

// Cell primitives from conserved values (utils.py:145-183 multiplies by the
// reciprocal of rho) and p, h (generic.py:27-87, 356-388).
template <typename T>
__device__ __forceinline__ void cons_to_prim(T rho, T ru, T rv, T rw, T re,
                                             T pe, T& u, T& v, T& w, T& e,
                                             T& p, T& h) {
  T inv = T(1) / rho;
  u = inv * ru;
  v = inv * rv;
  w = inv * rw;
  e = inv * re;
  T eint = e - T(0.5) * (u * u + v * v + w * w) - pe;
  p = K<T>::gm1() * rho * eint;
  h = e + p / rho;
}

// ---------------------------------------------------------------------------
// Face reconstruction. A stencil s[0 .. LO+RI-1] holds the cell values
// v[i-LO .. i+RI-1] around face i-1/2; neg comes from the left cell i-1,
// pos from the right cell i (compressible_navier_stokes.py:597-615).
// WENO-JS weights alpha_r = d_r / (eps + beta_r)^2 with eps = 1e-6 and the
// candidate polynomials of the reference prototype
// (demo/swirl_c_prototype.ipynb `weno5`, cell 4).
// ---------------------------------------------------------------------------
template <int SCHEME>
struct Stencil;

template <>
struct Stencil<0> {  // WENO5
  static constexpr int LO = 3, RI = 3;
};
template <>
struct Stencil<1> {  // WENO3
  static constexpr int LO = 2, RI = 2;
};
template <>
struct Stencil<2> {  // MUSCL
  static constexpr int LO = 2, RI = 2;
};
template <>
struct Stencil<3> {  // NODE (identity)
  static constexpr int LO = 0, RI = 1;
};

// WENO5 value on the right face (c+1/2) of cell c from v[c-2..c+2].
template <typename T>
__device__ __forceinline__ T weno5_right(T vm2, T vm1, T v0, T vp1, T vp2) {
  const T c1312 = T(13.0 / 12.0), q = T(0.25), eps = T(1e-6);
  T a = v0 - T(2) * vp1 + vp2, b = T(3) * v0 - T(4) * vp1 + vp2;
  T b0 = c1312 * a * a + q * b * b;
  a = vm1 - T(2) * v0 + vp1;
  b = vm1 - vp1;
  T b1 = c1312 * a * a + q * b * b;
  a = vm2 - T(2) * vm1 + v0;
  b = vm2 - T(4) * vm1 + T(3) * v0;
  T b2 = c1312 * a * a + q * b * b;
  b0 += eps;
  b1 += eps;
  b2 += eps;
  T a0 = T(0.3) * rcp_(b0 * b0);
  T a1 = T(0.6) * rcp_(b1 * b1);
  T a2 = T(0.1) * rcp_(b2 * b2);
  T q0 = T(1.0 / 3.0) * v0 + T(5.0 / 6.0) * vp1 - T(1.0 / 6.0) * vp2;
  T q1 = T(-1.0 / 6.0) * vm1 + T(5.0 / 6.0) * v0 + T(1.0 / 3.0) * vp1;
  T q2 = T(1.0 / 3.0) * vm2 - T(7.0 / 6.0) * vm1 + T(11.0 / 6.0) * v0;
  return (a0 * q0 + a1 * q1 + a2 * q2) * rcp_(a0 + a1 + a2);
}

// WENO5 value on the left face (c-1/2) of cell c from v[c-2..c+2].
template <typename T>
__device__ __forceinline__ T weno5_left(T vm2, T vm1, T v0, T vp1, T vp2) {
  const T c1312 = T(13.0 / 12.0), q = T(0.25), eps = T(1e-6);
  T a = v0 - T(2) * vp1 + vp2, b = T(3) * v0 - T(4) * vp1 + vp2;
  T b0 = c1312 * a * a + q * b * b;
  a = vm1 - T(2) * v0 + vp1;
  b = vm1 - vp1;
  T b1 = c1312 * a * a + q * b * b;
  a = vm2 - T(2) * vm1 + v0;
  b = vm2 - T(4) * vm1 + T(3) * v0;
  T b2 = c1312 * a * a + q * b * b;
  b0 += eps;
  b1 += eps;
  b2 += eps;
  T a0 = T(0.1) * rcp_(b0 * b0);
  T a1 = T(0.6) * rcp_(b1 * b1);
  T a2 = T(0.3) * rcp_(b2 * b2);
  T q0 = T(11.0 / 6.0) * v0 - T(7.0 / 6.0) * vp1 + T(1.0 / 3.0) * vp2;
  T q1 = T(1.0 / 3.0) * vm1 + T(5.0 / 6.0) * v0 - T(1.0 / 6.0) * vp1;
  T q2 = T(-1.0 / 6.0) * vm2 + T(5.0 / 6.0) * vm1 + T(1.0 / 3.0) * v0;
  return (a0 * q0 + a1 * q1 + a2 * q2) * rcp_(a0 + a1 + a2);
}

// WENO3 (k = 2) right / left face values of cell c from v[c-1..c+1], with
// d = (2/3, 1/3) and candidates c[-1..1] = (3/2,-1/2), (1/2,1/2), (-1/2,3/2).
template <typename T>
__device__ __forceinline__ T weno3_right(T vm1, T v0, T vp1) {
  const T eps = T(1e-6);
  T b0 = (vp1 - v0) * (vp1 - v0) + eps;
  T b1 = (v0 - vm1) * (v0 - vm1) + eps;
  T a0 = T(2.0 / 3.0) * rcp_(b0 * b0);
  T a1 = T(1.0 / 3.0) * rcp_(b1 * b1);
  T q0 = T(0.5) * v0 + T(0.5) * vp1;
  T q1 = T(-0.5) * vm1 + T(1.5) * v0;
  return (a0 * q0 + a1 * q1) * rcp_(a0 + a1);
}
template <typename T>
__device__ __forceinline__ T weno3_left(T vm1, T v0, T vp1) {
  const T eps = T(1e-6);
  T b0 = (vp1 - v0) * (vp1 - v0) + eps;
  T b1 = (v0 - vm1) * (v0 - vm1) + eps;
  T a0 = T(1.0 / 3.0) * rcp_(b0 * b0);
  T a1 = T(2.0 / 3.0) * rcp_(b1 * b1);
  T q0 = T(1.5) * v0 - T(0.5) * vp1;
  T q1 = T(0.5) * vm1 + T(0.5) * v0;
  return (a0 * q0 + a1 * q1) * rcp_(a0 + a1);
}

// MUSCL slope of cell c: phi(r) * dp with r = dnn(dm, dp).
template <typename T>
__device__ __forceinline__ T muscl_slope(T vm1, T v0, T vp1, int limiter) {
  T dp = vp1 - v0, dm = v0 - vm1;
  T r = dnn(dm, dp);
  T phi;
  if (limiter == 0) {  // van Leer
    // From |r| >= 2^54 (2^25 in single precision) 1 + |r| rounds to |r| and
    // the formula gives exactly 2 (r > 0) or 0 (r < 0); those values are
    // taken directly there, which also covers ratios where r + |r|
    // overflows or r is infinite (dp subnormal under dm: double precision
    // keeps subnormals), for which the formula gives inf or NaN.
    T a = abs_(r);
    const T big = sizeof(T) == 8 ? T(18014398509481984.0) : T(33554432.0);
    phi = a >= big ? (r > T(0) ? T(2) : T(0)) : (r + a) / (T(1) + a);
  } else if (limiter == 1) {  // monotonized central
    phi = max_(T(0), min_(min_(T(2) * r, T(0.5) * (T(1) + r)), T(2)));
  } else {  // minmod
    phi = max_(T(0), min_(r, T(1)));
  }
  return phi * dp;
}

// ---------------------------------------------------------------------------
// Cell-centred reconstruction: both face values of one cell c from its
// stencil s[0 .. CL+CR] = v[c-CL .. c+CR]. `right` is the neg value of face
// c+1/2, `left` the pos value of face c-1/2. For WENO the smoothness
// indicators and the reciprocals 1/(eps+beta_r)^2 are shared by both sides.
// NODE keeps the identity mock's convention (face i-1/2 takes v[i] on both
// sides), i.e. right(c) = v[c+1], left(c) = v[c].
// ---------------------------------------------------------------------------
template <int SCHEME>
struct CellStencil;
template <>
struct CellStencil<0> {
  static constexpr int CL = 2, CR = 2;
};
template <>
struct CellStencil<1> {
  static constexpr int CL = 1, CR = 1;
};
template <>
struct CellStencil<2> {
  static constexpr int CL = 1, CR = 1;
};
template <>
struct CellStencil<3> {
  static constexpr int CL = 0, CR = 1;
};

template <int SCHEME, typename T>
__device__ __forceinline__ void reconstruct_cell(const T* s, int limiter,
                                                 T& left, T& right) {
  if constexpr (SCHEME == 0) {
    const T vm2 = s[0], vm1 = s[1], v0 = s[2], vp1 = s[3], vp2 = s[4];
    const T c1312 = T(13.0 / 12.0), q = T(0.25), eps = T(1e-6);
    T a = v0 - T(2) * vp1 + vp2, b = T(3) * v0 - T(4) * vp1 + vp2;
    T b0 = c1312 * a * a + q * b * b;
    a = vm1 - T(2) * v0 + vp1;
    b = vm1 - vp1;
    T b1 = c1312 * a * a + q * b * b;
    a = vm2 - T(2) * vm1 + v0;
    b = vm2 - T(4) * vm1 + T(3) * v0;
    T b2 = c1312 * a * a + q * b * b;
    b0 += eps;
    b1 += eps;
    b2 += eps;
    const T i0 = rcp_(b0 * b0), i1 = rcp_(b1 * b1), i2 = rcp_(b2 * b2);
    {  // right face: d = (0.3, 0.6, 0.1)
      const T a0 = T(0.3) * i0, a1 = T(0.6) * i1, a2 = T(0.1) * i2;
      const T q0 = T(1.0 / 3.0) * v0 + T(5.0 / 6.0) * vp1 - T(1.0 / 6.0) * vp2;
      const T q1 = T(-1.0 / 6.0) * vm1 + T(5.0 / 6.0) * v0 + T(1.0 / 3.0) * vp1;
      const T q2 = T(1.0 / 3.0) * vm2 - T(7.0 / 6.0) * vm1 + T(11.0 / 6.0) * v0;
      right = (a0 * q0 + a1 * q1 + a2 * q2) * rcp_(a0 + a1 + a2);
    }
    {  // left face: d = (0.1, 0.6, 0.3)
      const T a0 = T(0.1) * i0, a1 = T(0.6) * i1, a2 = T(0.3) * i2;
      const T q0 = T(11.0 / 6.0) * v0 - T(7.0 / 6.0) * vp1 + T(1.0 / 3.0) * vp2;
      const T q1 = T(1.0 / 3.0) * vm1 + T(5.0 / 6.0) * v0 - T(1.0 / 6.0) * vp1;
      const T q2 = T(-1.0 / 6.0) * vm2 + T(5.0 / 6.0) * vm1 + T(1.0 / 3.0) * v0;
      left = (a0 * q0 + a1 * q1 + a2 * q2) * rcp_(a0 + a1 + a2);
    }
  } else if constexpr (SCHEME == 1) {
    const T vm1 = s[0], v0 = s[1], vp1 = s[2];
    const T eps = T(1e-6);
    T b0 = (vp1 - v0) * (vp1 - v0) + eps;
    T b1 = (v0 - vm1) * (v0 - vm1) + eps;
    const T i0 = rcp_(b0 * b0), i1 = rcp_(b1 * b1);
    {
      const T a0 = T(2.0 / 3.0) * i0, a1 = T(1.0 / 3.0) * i1;
      right = (a0 * (T(0.5) * v0 + T(0.5) * vp1) +
               a1 * (T(-0.5) * vm1 + T(1.5) * v0)) * rcp_(a0 + a1);
    }
    {
      const T a0 = T(1.0 / 3.0) * i0, a1 = T(2.0 / 3.0) * i1;
      left = (a0 * (T(1.5) * v0 - T(0.5) * vp1) +
              a1 * (T(0.5) * vm1 + T(0.5) * v0)) * rcp_(a0 + a1);
    }
  } else if constexpr (SCHEME == 2) {
    const T sl = muscl_slope(s[0], s[1], s[2], limiter);
    right = s[1] + T(0.5) * sl;
    left = s[1] - T(0.5) * sl;
  } else {
    left = s[0];
    right = s[1];
  }
}

// ---------------------------------------------------------------------------
// Packed single-precision reconstruction. The neg value of face i-1/2 (right
// face of cell i-1) and its pos value (left face of cell i) use the same
// formulas on stencils shifted by one cell, with mirrored coefficients, so
// both run as one sequence of Blackwell f32x2 instructions (FFMA2 / FADD2 /
// FMUL2): lane x = neg, lane y = pos.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  return __ffma2_rn(a, b, c);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 rcp2(float2 a) {
  return make_float2(1.0f / a.x, 1.0f / a.y);
}

// WENO5-JS pair from the 6-cell stencil s[0..5] = v[i-3..i+2].
__device__ __forceinline__ float2 weno5_pair(const float* s) {
  const float2 vm2 = f2(s[0], s[1]), vm1 = f2(s[1], s[2]), v0 = f2(s[2], s[3]);
  const float2 vp1 = f2(s[3], s[4]), vp2 = f2(s[4], s[5]);
  const float2 k1312 = f2(13.0f / 12.0f, 13.0f / 12.0f);
  const float2 kq = f2(0.25f, 0.25f), eps = f2(1e-6f, 1e-6f);
  const float2 m2 = f2(-2.0f, -2.0f), k3 = f2(3.0f, 3.0f), m4 = f2(-4.0f, -4.0f);
  // beta_0 on (v0, vp1, vp2)
  float2 a = add2(fma2(m2, vp1, v0), vp2);
  float2 b = fma2(m4, vp1, fma2(k3, v0, vp2));
  float2 b0 = fma2(mul2(k1312, a), a, mul2(mul2(kq, b), b));
  // beta_1 on (vm1, v0, vp1)
  a = add2(fma2(m2, v0, vm1), vp1);
  b = add2(vm1, mul2(f2(-1.0f, -1.0f), vp1));
  float2 b1 = fma2(mul2(k1312, a), a, mul2(mul2(kq, b), b));
  // beta_2 on (vm2, vm1, v0)
  a = add2(fma2(m2, vm1, vm2), v0);
  b = fma2(k3, v0, fma2(m4, vm1, vm2));
  float2 b2 = fma2(mul2(k1312, a), a, mul2(mul2(kq, b), b));
  b0 = add2(b0, eps);
  b1 = add2(b1, eps);
  b2 = add2(b2, eps);
  // alpha_r = d_r / (eps + beta_r)^2; d = (0.3, 0.6, 0.1) for neg and the
  // mirror (0.1, 0.6, 0.3) for pos.
  const float2 a0 = mul2(f2(0.3f, 0.1f), rcp2(mul2(b0, b0)));
  const float2 a1 = mul2(f2(0.6f, 0.6f), rcp2(mul2(b1, b1)));
  const float2 a2 = mul2(f2(0.1f, 0.3f), rcp2(mul2(b2, b2)));
  // Candidates: neg = right face of the cell, pos = left face.
  const float2 q0 = fma2(f2(-1.0f / 6.0f, 1.0f / 3.0f), vp2,
                         fma2(f2(5.0f / 6.0f, -7.0f / 6.0f), vp1,
                              mul2(f2(1.0f / 3.0f, 11.0f / 6.0f), v0)));
  const float2 q1 = fma2(f2(1.0f / 3.0f, -1.0f / 6.0f), vp1,
                         fma2(f2(5.0f / 6.0f, 5.0f / 6.0f), v0,
                              mul2(f2(-1.0f / 6.0f, 1.0f / 3.0f), vm1)));
  const float2 q2 = fma2(f2(11.0f / 6.0f, 1.0f / 3.0f), v0,
                         fma2(f2(-7.0f / 6.0f, 5.0f / 6.0f), vm1,
                              mul2(f2(1.0f / 3.0f, -1.0f / 6.0f), vm2)));
  const float2 num = fma2(a2, q2, fma2(a1, q1, mul2(a0, q0)));
  const float2 den = add2(add2(a0, a1), a2);
  return mul2(num, rcp2(den));
}

// WENO3-JS pair from s[0..3] = v[i-2..i+1].
__device__ __forceinline__ float2 weno3_pair(const float* s) {
  const float2 vm1 = f2(s[0], s[1]), v0 = f2(s[1], s[2]), vp1 = f2(s[2], s[3]);
  const float2 eps = f2(1e-6f, 1e-6f);
  float2 d0 = add2(vp1, mul2(f2(-1.0f, -1.0f), v0));
  float2 d1 = add2(v0, mul2(f2(-1.0f, -1.0f), vm1));
  float2 b0 = fma2(d0, d0, eps), b1 = fma2(d1, d1, eps);
  const float2 a0 = mul2(f2(2.0f / 3.0f, 1.0f / 3.0f), rcp2(mul2(b0, b0)));
  const float2 a1 = mul2(f2(1.0f / 3.0f, 2.0f / 3.0f), rcp2(mul2(b1, b1)));
  const float2 q0 = fma2(f2(0.5f, -0.5f), vp1, mul2(f2(0.5f, 1.5f), v0));
  const float2 q1 = fma2(f2(1.5f, 0.5f), v0, mul2(f2(-0.5f, 0.5f), vm1));
  return mul2(fma2(a1, q1, mul2(a0, q0)), rcp2(add2(a0, a1)));
}

template <int SCHEME, typename T>
__device__ __forceinline__ void reconstruct(const T* s, int limiter, T& neg,
                                            T& pos) {
  if constexpr (SCHEME == 0) {
    if constexpr (sizeof(T) == 4 && SWC_PACKED_WENO) {
      float2 r = weno5_pair(s);
      neg = r.x;
      pos = r.y;
    } else {
      neg = weno5_right(s[0], s[1], s[2], s[3], s[4]);
      pos = weno5_left(s[1], s[2], s[3], s[4], s[5]);
    }
  } else if constexpr (SCHEME == 1) {
    if constexpr (sizeof(T) == 4 && SWC_PACKED_WENO) {
      float2 r = weno3_pair(s);
      neg = r.x;
      pos = r.y;
    } else {
      neg = weno3_right(s[0], s[1], s[2]);
      pos = weno3_left(s[1], s[2], s[3]);
    }
  } else if constexpr (SCHEME == 2) {
    neg = s[1] + T(0.5) * muscl_slope(s[0], s[1], s[2], limiter);
    pos = s[2] - T(0.5) * muscl_slope(s[1], s[2], s[3], limiter);
  } else {
    neg = s[0];
    pos = s[0];
  }
}

// ---------------------------------------------------------------------------
// Riemann solvers.
// ---------------------------------------------------------------------------
// Physical flux along D of one face state (compressible_navier_stokes.py:
// 338-427): mass m = rho*u_D; momentum m*u_i (+ p_upd when i == D); energy
// m*(e + p/rho) with the full p.
template <typename T, int D>
__device__ __forceinline__ void physical_flux(const Prim<T>& q, T p_upd,
                                              T* f) {
  T m = q.r * q.u[D];
  f[0] = m;
#pragma unroll
  for (int i = 0; i < 3; ++i) f[1 + i] = m * q.u[i];
  f[1 + D] = f[1 + D] + p_upd;
  f[4] = m * (q.e + q.p / q.r);
}

// Roe-averaged wave-speed estimates (hll.py:178-283): c = sqrt(gamma p/rho)
// per side, Roe averages with sqrt(rho) weights and reciprocal_no_nan,
// c~ from the sensible enthalpy with the potential energy pe of the cell at
// the face index (generic.py:144-148, 391-423).
template <typename T, int D>
__device__ __forceinline__ void hll_speeds(const Prim<T>& l, const Prim<T>& r,
                                           T pe, T& s_l, T& s_r) {
  T c_l = sqrt_(K<T>::gamma() * l.p / l.r);
  T c_r = sqrt_(K<T>::gamma() * r.p / r.r);
  T rl = sqrt_(l.r), rr = sqrt_(r.r);
  T den = rl + rr;
  T inv = den == T(0) ? T(0) : T(1) / den;
  // Roe averages without FMA contraction: mirror-image states give exactly
  // u~ = 0 (hll.py:243-261 evaluates them as separate products).
  T ru[3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
    ru[i] = (mul_rn(rl, l.u[i]) + mul_rn(rr, r.u[i])) * inv;
  T rh = (mul_rn(rl, l.h) + mul_rn(rr, r.h)) * inv;
  T hs = rh - T(0.5) * (ru[0] * ru[0] + ru[1] * ru[1] + ru[2] * ru[2]) - pe;
  T rc = sqrt_(K<T>::gm1() * hs);
  s_l = min_(l.u[D] - c_l, ru[D] - rc);
  s_r = max_(r.u[D] + c_r, ru[D] + rc);
}

// HLL flux (hll.py:107-170): F = t1 F_R + t2 F_L - t3 (U_R - U_L). The wave
// speeds use the full pressure; pdl / pdr replace p in the aligned momentum
// flux when the helper variable p_dyn is present
// (compressible_navier_stokes.py:378).
template <typename T, int D>
__device__ __forceinline__ void hll_flux(const Prim<T>& l, const Prim<T>& r,
                                         T pdl, T pdr, T pe, T* f) {
  T s_l, s_r;
  hll_speeds<T, D>(l, r, pe, s_l, s_r);
  T ds = s_r - s_l;
  T t1 = dnn(min_(s_r, T(0)) - min_(s_l, T(0)), ds);
  T t2 = T(1) - t1;
  T t3 = dnn(s_r * abs_(s_l) - s_l * abs_(s_r), T(2) * ds);
  T fl[5], fr[5];
  physical_flux<T, D>(l, pdl, fl);
  physical_flux<T, D>(r, pdr, fr);
  T ul[5] = {l.r, mul_rn(l.r, l.u[0]), mul_rn(l.r, l.u[1]),
             mul_rn(l.r, l.u[2]), mul_rn(l.r, l.e)};
  T ur[5] = {r.r, mul_rn(r.r, r.u[0]), mul_rn(r.r, r.u[1]),
             mul_rn(r.r, r.u[2]), mul_rn(r.r, r.e)};
#pragma unroll
  for (int k = 0; k < 5; ++k)
    f[k] = t1 * fr[k] + t2 * fl[k] - t3 * (ur[k] - ul[k]);
}

// HLLC contact speed (hllc.py:328-341), zeroed when |s_m| < 1e-6.
template <typename T, int D>
__device__ __forceinline__ T hllc_contact(const Prim<T>& l, const Prim<T>& r,
                                          T s_l, T s_r) {
  T vl = l.u[D], vr = r.u[D];
  T num = (r.p - l.p) + mul_rn(mul_rn(l.r, vl), s_l - vl) -
          mul_rn(mul_rn(r.r, vr), s_r - vr);
  T den = mul_rn(l.r, s_l - vl) - mul_rn(r.r, s_r - vr);
  T s_m = dnn(num, den);
  return abs_(s_m) < T(1e-6) ? T(0) : s_m;
}

// HLLC flux (hllc.py:105-257). With p_dyn present, the wave speeds and the
// star states use p = p_dyn (hllc.py:109-120) while the physical flux keeps
// the full p in the energy flux. The four-way select of hllc.py:229-243
// picks one side k and whether its star flux applies; only that side's flux
// is evaluated (same value as evaluating all four and selecting).
template <typename T, int D>
__device__ __forceinline__ void hllc_flux(const Prim<T>& l, const Prim<T>& r,
                                          T pdl, T pdr, T pe, T* f) {
  Prim<T> lu = l, ru = r;
  lu.p = pdl;
  ru.p = pdr;
  T s_l, s_r;
  hll_speeds<T, D>(lu, ru, pe, s_l, s_r);
  T s_m = hllc_contact<T, D>(lu, ru, s_l, s_r);
  bool c1 = s_l >= T(0);
  bool c2 = (s_l <= T(0)) && (s_m >= T(0));
  bool c3 = (s_m <= T(0)) && (s_r >= T(0));
  bool left = c1 || c2;
  bool star = !c1 && (c2 || c3);
  Prim<T> q;
  q.r = left ? l.r : r.r;
#pragma unroll
  for (int i = 0; i < 3; ++i) q.u[i] = left ? l.u[i] : r.u[i];
  q.e = left ? l.e : r.e;
  q.p = left ? l.p : r.p;
  q.h = left ? l.h : r.h;
  T pd = left ? pdl : pdr;
  T s_k = left ? s_l : s_r;
  physical_flux<T, D>(q, pd, f);
  if (star) {
    T v_k = q.u[D];
    T rat = dnn(s_k, s_k - s_m);
    T dv = s_m - v_k;
    f[0] = f[0] + q.r * dv * rat;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (i == D) {
        f[1 + i] = f[1 + i] + q.r * s_k * (dnn(s_k - v_k, s_k - s_m) * s_m - v_k);
      } else {
        f[1 + i] = f[1 + i] + q.r * dv * q.u[i] * rat;
      }
    }
    f[4] = f[4] + q.r * rat * dv * (q.e + pd / q.r + (s_k - v_k) * s_m);
  }
}

template <int RIEMANN, typename T, int D>
__device__ __forceinline__ void riemann(const Prim<T>& l, const Prim<T>& r,
                                        T pe, T* f) {
  if constexpr (RIEMANN == 0) {
    hll_flux<T, D>(l, r, l.p, r.p, pe, f);
  } else {
    hllc_flux<T, D>(l, r, l.p, r.p, pe, f);
  }
}

// Fluxes of `ns` transported scalars phi_k with face values phl/phr: the
// generic branches of the physical flux (m*phi,
// compressible_navier_stokes.py:419-427), of HLL (hll.py:159-170) and of the
// HLLC star flux (hllc.py:182-192; wave speeds from the p_dyn-updated states,
// hllc.py:105-120).
template <int RIEMANN, typename T, int D>
__device__ __forceinline__ void scalar_fluxes(const Prim<T>& l,
                                              const Prim<T>& r, T pdl, T pdr,
                                              T pe, int ns, const T* phl,
                                              const T* phr, T* out) {
  const T ml = l.r * l.u[D], mr = r.r * r.u[D];
  if constexpr (RIEMANN == 0) {
    T s_l, s_r;
    hll_speeds<T, D>(l, r, pe, s_l, s_r);
    T ds = s_r - s_l;
    T t1 = dnn(min_(s_r, T(0)) - min_(s_l, T(0)), ds);
    T t2 = T(1) - t1;
    T t3 = dnn(s_r * abs_(s_l) - s_l * abs_(s_r), T(2) * ds);
#pragma unroll
    for (int k = 0; k < ns; ++k)
      out[k] = t1 * (mr * phr[k]) + t2 * (ml * phl[k]) -
               t3 * (mul_rn(r.r, phr[k]) - mul_rn(l.r, phl[k]));
  } else {
    Prim<T> lu = l, ru = r;
    lu.p = pdl;
    ru.p = pdr;
    T s_l, s_r;
    hll_speeds<T, D>(lu, ru, pe, s_l, s_r);
    T s_m = hllc_contact<T, D>(lu, ru, s_l, s_r);
    bool c1 = s_l >= T(0);
    bool c2 = (s_l <= T(0)) && (s_m >= T(0));
    bool c3 = (s_m <= T(0)) && (s_r >= T(0));
    bool left = c1 || c2;
    bool star = !c1 && (c2 || c3);
    const Prim<T>& q = left ? l : r;
    T s_k = left ? s_l : s_r;
    T m = left ? ml : mr;
#pragma unroll
    for (int k = 0; k < ns; ++k) {
      T ph = left ? phl[k] : phr[k];
      T fk = m * ph;
      if (star) fk = fk + q.r * (s_m - q.u[D]) * ph * dnn(s_k, s_k - s_m);
      out[k] = fk;
    }
  }
}

// ---------------------------------------------------------------------------
// Viscous flux on the face between cells a (i-1) and b (i) along D
// (compressible_navier_stokes.py:618-707; diffusion.py:33-109;
// fluid.py:31-111). `ga[t][c]` / `gb[t][c]` are the central differences
// (f[+1]-f[-1])/(2h_t) of velocity component c along tangential axis t at
// cells a and b; only c == t and c == D are used.
// ---------------------------------------------------------------------------
template <typename T, int D>
__device__ __forceinline__ void viscous_flux(
    T ra, T rb, const T* ua, const T* ub, T pa, T pb, const T ga[3][3],
    const T gb[3][3], T h_d, T nu, T inv_pr, T* f) {
  // Backward differences along D of u, v, w and T = p/(rho R).
  T bd[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) bd[c] = (ub[c] - ua[c]) / h_d;
  // div on face D: bwd_D(u_D) + sum over t != D of lin(central_t(u_t)).
  T g[3];  // g[c] = d u_c / d x_c on face D
#pragma unroll
  for (int c = 0; c < 3; ++c)
    g[c] = (c == D) ? bd[D] : T(0.5) * (ga[c][c] + gb[c][c]);
  T div = g[0] + g[1] + g[2];
  T rf = T(0.5) * (ra + rb);
  T tau[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    T s;
    if (c == D) {
      s = bd[D] - T(1.0 / 3.0) * div;
    } else {
      // s_cD = 0.5 * (bwd_D(u_c) + lin_D(central_c(u_D)))
      s = T(0.5) * (bd[c] + T(0.5) * (ga[c][D] + gb[c][D]));
    }
    tau[c] = T(2) * rf * nu * s;
  }
  T uf[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) uf[c] = T(0.5) * (ua[c] + ub[c]);
  T ta = pa / (ra * K<T>::r_gas());
  T tb = pb / (rb * K<T>::r_gas());
  T ka = inv_pr * K<T>::cp() * (nu * ra);
  T kb = inv_pr * K<T>::cp() * (nu * rb);
  T q = -(T(0.5) * (ka + kb)) * ((tb - ta) / h_d);
  T dot = uf[0] * tau[0] + uf[1] * tau[1] + uf[2] * tau[2];
#pragma unroll
  for (int c = 0; c < 3; ++c) f[1 + c] = f[1 + c] + (-tau[c]);
  f[4] = f[4] + (q + (-dot));
}

}  // namespace swc
