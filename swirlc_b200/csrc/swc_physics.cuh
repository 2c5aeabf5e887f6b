// Device-side physics of the Swirl-C compressible RHS, shared by the fused
// stage kernel and the unit-level kernels.
//
// Each function states the reference lines it follows (paths relative to the
// swirl_c project root). Arithmetic runs in T (float or double).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

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
// x / y by a divisor y fixed for the whole launch, with ry = rcp_(y) formed
// once: the single-precision quotient under -use_fast_math is x * (1/y) with
// the hardware reciprocal, i.e. this product; double precision keeps the
// correctly rounded quotient.
__device__ __forceinline__ float divk(float x, float /*y*/, float ry) { return x * ry; }
__device__ __forceinline__ double divk(double x, double y, double /*ry*/) { return x / y; }
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
// Finite test on the exponent bits (unaffected by fast-math flags).
__device__ __forceinline__ bool finite_(float a) {
  return (__float_as_uint(a) & 0x7f800000u) != 0x7f800000u;
}
__device__ __forceinline__ bool finite_(double a) {
  return (static_cast<unsigned long long>(__double_as_longlong(a)) &
          0x7ff0000000000000ull) != 0x7ff0000000000000ull;
}
// CFL limit of one cell as it enters the min-reduction: delta_d/(|u_d|+c),
// or 0 when rho, p or rho_e is not finite or the limit itself is NaN
// (p/rho < 0). 0 is never a limit of a finite state, so a reduced minimum of
// 0 reports a non-finite or unphysical state to the host
// (swc_clock_status).
template <typename T>
__device__ __forceinline__ double cfl_limit_or_flag(T rho, T p, T rhoe, T l) {
  const bool ok = finite_(rho) && finite_(p) && finite_(rhoe) && (l == l);
  return ok ? double(l) : 0.0;
}

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

// MUSCL slope of cell c for the monotonized-central (1) and minmod (2)
// limiters: phi(r) * dp with r = dnn(dm, dp); or (limiter 3) the reference
// prototype's slope (demo/swirl_c_prototype.ipynb `muscl`, cell 4): minmod
// of the central difference (v[c+1] - v[c-1]) / 4, the forward and the
// backward difference, i.e. the smallest magnitude of the three where all
// three have the same sign, else 0. The van Leer limiter (0) is formed lane
// by lane in muscl_slope_v.
template <typename T>
__device__ __forceinline__ T muscl_slope(T vm1, T v0, T vp1, int limiter) {
  T dp = vp1 - v0, dm = v0 - vm1;
  if (limiter == 3) {
    const T c2 = (vp1 - vm1) * T(0.25);
    const T m = min_(min_(abs_(c2), abs_(dp)), abs_(dm));
    const bool up = c2 > T(0) && dp > T(0) && dm > T(0);
    const bool down = c2 < T(0) && dp < T(0) && dm < T(0);
    return up ? m : (down ? -m : T(0));
  }
  T r = dnn(dm, dp);
  T phi;
  if (limiter == 1) {  // monotonized central
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

// ---------------------------------------------------------------------------
// Lane-generic reconstruction used by the fused stage. Face reconstruction
// applies the same formulas to every variable on the same stencil cells, so
// two variables share one instruction stream: Two<float> runs them as
// Blackwell f32x2 instructions (FFMA2 / FADD2 / FMUL2 issue both lanes in one
// slot), Two<double> as two scalar lanes, One<T> is a single variable. Every
// product and sum is rounded as written (no contraction), so a value comes
// out bit for bit the same whichever lane count, call site or form (face
// pair or cell-centred) computes it. Reciprocals run per lane.
// ---------------------------------------------------------------------------
template <typename T>
struct One;
template <>
struct One<float> {
  using S = float;
  using V = float;
  static __device__ __forceinline__ V splat(float a) { return a; }
  static __device__ __forceinline__ V fma(V a, V b, V c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ V mul(V a, V b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ V add(V a, V b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ V sub(V a, V b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ V rcp(V a) { return 1.0f / a; }
  // a / b as a times the reciprocal of b (what the fast-math quotient is).
  static __device__ __forceinline__ V div(V a, V b) { return __fmul_rn(a, 1.0f / b); }
  // x where p > 0, else 0.
  static __device__ __forceinline__ V sel_pos(V p, V x) { return p > 0.0f ? x : 0.0f; }
  template <class F>
  static __device__ __forceinline__ V map3(F f, V a, V b, V c) { return f(a, b, c); }
};
template <>
struct One<double> {
  using S = double;
  using V = double;
  static __device__ __forceinline__ V splat(double a) { return a; }
  static __device__ __forceinline__ V fma(V a, V b, V c) { return __fma_rn(a, b, c); }
  static __device__ __forceinline__ V mul(V a, V b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ V add(V a, V b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ V sub(V a, V b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ V rcp(V a) { return 1.0 / a; }
  static __device__ __forceinline__ V div(V a, V b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ V sel_pos(V p, V x) { return p > 0.0 ? x : 0.0; }
  template <class F>
  static __device__ __forceinline__ V map3(F f, V a, V b, V c) { return f(a, b, c); }
};
template <typename T>
struct Two;
template <>
struct Two<float> {
  using S = float;
  using V = float2;
  static __device__ __forceinline__ V mk(float a, float b) { return make_float2(a, b); }
  static __device__ __forceinline__ V splat(float a) { return make_float2(a, a); }
  static __device__ __forceinline__ V fma(V a, V b, V c) { return __ffma2_rn(a, b, c); }
  static __device__ __forceinline__ V mul(V a, V b) { return __fmul2_rn(a, b); }
  static __device__ __forceinline__ V add(V a, V b) { return __fadd2_rn(a, b); }
  // a - b, rounded once (b * -1 is exact).
  static __device__ __forceinline__ V sub(V a, V b) { return __ffma2_rn(b, splat(-1.0f), a); }
  static __device__ __forceinline__ V rcp(V a) { return make_float2(1.0f / a.x, 1.0f / a.y); }
  static __device__ __forceinline__ V div(V a, V b) { return __fmul2_rn(a, rcp(b)); }
  static __device__ __forceinline__ V sel_pos(V p, V x) {
    return make_float2(p.x > 0.0f ? x.x : 0.0f, p.y > 0.0f ? x.y : 0.0f);
  }
  template <class F>
  static __device__ __forceinline__ V map3(F f, V a, V b, V c) {
    return make_float2(f(a.x, b.x, c.x), f(a.y, b.y, c.y));
  }
};
template <>
struct Two<double> {
  using S = double;
  using V = double2;
  static __device__ __forceinline__ V mk(double a, double b) { return make_double2(a, b); }
  static __device__ __forceinline__ V splat(double a) { return make_double2(a, a); }
  static __device__ __forceinline__ V fma(V a, V b, V c) {
    return make_double2(__fma_rn(a.x, b.x, c.x), __fma_rn(a.y, b.y, c.y));
  }
  static __device__ __forceinline__ V mul(V a, V b) {
    return make_double2(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
  }
  static __device__ __forceinline__ V add(V a, V b) {
    return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
  }
  static __device__ __forceinline__ V sub(V a, V b) {
    return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
  }
  static __device__ __forceinline__ V rcp(V a) { return make_double2(1.0 / a.x, 1.0 / a.y); }
  static __device__ __forceinline__ V div(V a, V b) {
    return make_double2(__ddiv_rn(a.x, b.x), __ddiv_rn(a.y, b.y));
  }
  static __device__ __forceinline__ V sel_pos(V p, V x) {
    return make_double2(p.x > 0.0 ? x.x : 0.0, p.y > 0.0 ? x.y : 0.0);
  }
  template <class F>
  static __device__ __forceinline__ V map3(F f, V a, V b, V c) {
    return make_double2(f(a.x, b.x, c.x), f(a.y, b.y, c.y));
  }
};

// WENO5-JS on the cell stencil v[c-2..c+2]: alpha_r = d_r / (eps + beta_r)^2
// with eps = 1e-6, the smoothness indicators
// beta_r = 13/12 a_r^2 + 1/4 b_r^2 and the candidate polynomials q_r of the
// reference prototype's `weno5`; the value is sum alpha_r q_r / sum alpha_r.
// Computed as: B_r = 4 (beta_r + eps) = 13/3 a_r^2 + (b_r^2 + 4 eps) (eps
// folds into an FMA; a_r, b_r from first differences, below),
// i_r = 1/B_r^2 (shared by both faces of the cell), and
// per face num = sum i_r (d_r q_r), den = sum d_r i_r with d_r folded into
// the candidates' coefficients. The common factor 1/16 of i_r cancels in
// num/den, so the weights are the prototype's in exact arithmetic.
// Right face (c+1/2): d = (0.3, 0.6, 0.1); left face (c-1/2): d mirrored.
template <class O>
struct Weno5Inv {
  typename O::V i0, i1, i2;
};
// The indicators are built from the first differences e_k = v[k+1] - v[k]
// of the stencil: a_r is the second difference of candidate r's three cells
// (e_hi - e_lo), so two neighbouring cells' indicators share two of their
// three (a_r, 13/3 a_r) pairs; b_r = e_hi - 3 e_lo (r = 0), e_lo + e_hi
// (r = 1) and e_lo - 3 e_hi (r = 2) up to sign.
template <class O>
struct Weno5Tri {  // second difference a of three cells and 13/3 a
  typename O::V a, ca;
};
template <class O>
__device__ __forceinline__ Weno5Tri<O> weno5_tri(typename O::V e_lo,
                                                 typename O::V e_hi) {
  using S = typename O::S;
  const typename O::V a = O::sub(e_hi, e_lo);
  return {a, O::mul(O::splat(S(13.0 / 3.0)), a)};
}
// 4 (beta + eps) = 13/3 a^2 + (b^2 + 4 eps).
template <class O>
__device__ __forceinline__ typename O::V weno5_b4(const Weno5Tri<O>& t,
                                                  typename O::V b) {
  using S = typename O::S;
  return O::fma(t.ca, t.a, O::fma(b, b, O::splat(S(4e-6))));
}
// Cell with differences dm2 = v[c-1]-v[c-2], dm1 = v[c]-v[c-1],
// d0 = v[c+1]-v[c], d1 = v[c+2]-v[c+1] and the second differences
// t2 = (dm2, dm1), t1 = (dm1, d0), t0 = (d0, d1).
template <class O>
__device__ __forceinline__ Weno5Inv<O> weno5_inv(
    const Weno5Tri<O>& t2, const Weno5Tri<O>& t1, const Weno5Tri<O>& t0,
    typename O::V dm2, typename O::V dm1, typename O::V d0,
    typename O::V d1) {
  using S = typename O::S;
  const typename O::V m3 = O::splat(S(-3));
  const typename O::V b0 = weno5_b4<O>(t0, O::fma(m3, d0, d1));
  const typename O::V b1 = weno5_b4<O>(t1, O::add(d0, dm1));
  const typename O::V b2 = weno5_b4<O>(t2, O::fma(m3, dm1, dm2));
  return {O::rcp(O::mul(b0, b0)), O::rcp(O::mul(b1, b1)),
          O::rcp(O::mul(b2, b2))};
}
// sum i_r dq_r / sum d_r i_r for the weighted candidates dq_r = d_r q_r.
template <class O>
__device__ __forceinline__ typename O::V weno5_combine(
    const Weno5Inv<O>& w, typename O::S d0, typename O::S d1,
    typename O::S d2, typename O::V dq0, typename O::V dq1,
    typename O::V dq2) {
  const typename O::V num =
      O::fma(w.i2, dq2, O::fma(w.i1, dq1, O::mul(w.i0, dq0)));
  const typename O::V den =
      O::fma(O::splat(d2), w.i2,
             O::fma(O::splat(d1), w.i1, O::mul(O::splat(d0), w.i0)));
  return O::mul(num, O::rcp(den));
}
template <class O>
__device__ __forceinline__ typename O::V weno5_right_v(
    const Weno5Inv<O>& w, typename O::V vm2, typename O::V vm1,
    typename O::V v0, typename O::V vp1, typename O::V vp2) {
  using S = typename O::S;
  using V = typename O::V;
  // 0.3 q0, 0.6 q1, 0.1 q2 with q0 = (2 v0 + 5 vp1 - vp2) / 6,
  // q1 = (-vm1 + 5 v0 + 2 vp1) / 6, q2 = (2 vm2 - 7 vm1 + 11 v0) / 6.
  const V dq0 = O::fma(O::splat(S(-0.05)), vp2,
                       O::fma(O::splat(S(0.25)), vp1,
                              O::mul(O::splat(S(0.1)), v0)));
  const V dq1 = O::fma(O::splat(S(0.2)), vp1,
                       O::fma(O::splat(S(0.5)), v0,
                              O::mul(O::splat(S(-0.1)), vm1)));
  const V dq2 = O::fma(O::splat(S(11.0 / 60.0)), v0,
                       O::fma(O::splat(S(-7.0 / 60.0)), vm1,
                              O::mul(O::splat(S(1.0 / 30.0)), vm2)));
  return weno5_combine<O>(w, S(0.3), S(0.6), S(0.1), dq0, dq1, dq2);
}
template <class O>
__device__ __forceinline__ typename O::V weno5_left_v(
    const Weno5Inv<O>& w, typename O::V vm2, typename O::V vm1,
    typename O::V v0, typename O::V vp1, typename O::V vp2) {
  using S = typename O::S;
  using V = typename O::V;
  // 0.1 q0, 0.6 q1, 0.3 q2 with q0 = (11 v0 - 7 vp1 + 2 vp2) / 6,
  // q1 = (2 vm1 + 5 v0 - vp1) / 6, q2 = (-vm2 + 5 vm1 + 2 v0) / 6.
  const V dq0 = O::fma(O::splat(S(1.0 / 30.0)), vp2,
                       O::fma(O::splat(S(-7.0 / 60.0)), vp1,
                              O::mul(O::splat(S(11.0 / 60.0)), v0)));
  const V dq1 = O::fma(O::splat(S(-0.1)), vp1,
                       O::fma(O::splat(S(0.5)), v0,
                              O::mul(O::splat(S(0.2)), vm1)));
  const V dq2 = O::fma(O::splat(S(0.1)), v0,
                       O::fma(O::splat(S(0.25)), vm1,
                              O::mul(O::splat(S(-0.05)), vm2)));
  return weno5_combine<O>(w, S(0.1), S(0.6), S(0.3), dq0, dq1, dq2);
}

// WENO3 (k = 2) on v[c-1..c+1]: reciprocals of (eps + beta_r)^2, then the
// right face (d = (2/3, 1/3), candidates (1/2, 1/2) and (-1/2, 3/2)) or the
// left face (d mirrored).
template <class O>
__device__ __forceinline__ void weno3_inv(typename O::V vm1, typename O::V v0,
                                          typename O::V vp1, typename O::V& i0,
                                          typename O::V& i1) {
  using S = typename O::S;
  using V = typename O::V;
  const V d0 = O::sub(vp1, v0), d1 = O::sub(v0, vm1);
  const V eps = O::splat(S(1e-6));
  const V b0 = O::add(O::mul(d0, d0), eps), b1 = O::add(O::mul(d1, d1), eps);
  i0 = O::rcp(O::mul(b0, b0));
  i1 = O::rcp(O::mul(b1, b1));
}
template <class O>
__device__ __forceinline__ typename O::V weno3_side_v(
    typename O::V i0, typename O::V i1, typename O::V vm1, typename O::V v0,
    typename O::V vp1, bool right) {
  using S = typename O::S;
  using V = typename O::V;
  const V h = O::splat(S(0.5)), mh = O::splat(S(-0.5)), k15 = O::splat(S(1.5));
  const V a0 = O::mul(O::splat(right ? S(2.0 / 3.0) : S(1.0 / 3.0)), i0);
  const V a1 = O::mul(O::splat(right ? S(1.0 / 3.0) : S(2.0 / 3.0)), i1);
  const V q0 = right ? O::fma(h, vp1, O::mul(h, v0)) : O::fma(mh, vp1, O::mul(k15, v0));
  const V q1 = right ? O::fma(k15, v0, O::mul(mh, vm1)) : O::fma(h, v0, O::mul(h, vm1));
  return O::mul(O::fma(a1, q1, O::mul(a0, q0)), O::rcp(O::add(a0, a1)));
}

// MUSCL slopes per lane (muscl_slope).
template <class O>
__device__ __forceinline__ typename O::V muscl_slope_v(typename O::V vm1,
                                                       typename O::V v0,
                                                       typename O::V vp1,
                                                       int limiter) {
  using S = typename O::S;
  if (limiter == 0) {
    // van Leer: phi(r) dp = (r + |r|) / (1 + |r|) dp with r = dm / dp is, in
    // exact arithmetic, the harmonic mean 2 dm dp / (dm + dp) where dm and
    // dp have the same sign (dm dp > 0) and 0 elsewhere (dp = 0 or dm = 0
    // included, as divide_no_nan gives r = 0 there). It is formed as
    // 2 dm * (dp / (dm + dp)): one quotient instead of two, no ratio r and
    // no product that can overflow (dp / (dm + dp) lies in (0, 1]), so
    // extreme ratios beside subnormal values (double precision keeps them)
    // need no special case; every lane op is a paired one where O pairs.
    const typename O::V dp = O::sub(vp1, v0), dm = O::sub(v0, vm1);
    const typename O::V q = O::div(dp, O::add(dm, dp));
    return O::sel_pos(O::mul(dm, dp), O::mul(O::add(dm, dm), q));
  }
  return O::map3([limiter](S a, S b, S c) { return muscl_slope(a, b, c, limiter); },
                 vm1, v0, vp1);
}

// Face i-1/2 from s[k] = v[i-LO+k] (Stencil<SCHEME>): neg from cell i-1
// (its right face), pos from cell i (its left face).
template <int SCHEME, class O>
__device__ __forceinline__ void recon_face(const typename O::V* s, int limiter,
                                           typename O::V& neg,
                                           typename O::V& pos) {
  using S = typename O::S;
  if constexpr (SCHEME == 0) {
    // Cells i-1 (s[0..4]) and i (s[1..5]) share the differences e1..e3
    // and the second differences f1, f2.
    typename O::V e[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) e[k] = O::sub(s[k + 1], s[k]);
    Weno5Tri<O> f[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) f[k] = weno5_tri<O>(e[k], e[k + 1]);
    neg = weno5_right_v<O>(
        weno5_inv<O>(f[0], f[1], f[2], e[0], e[1], e[2], e[3]), s[0], s[1],
        s[2], s[3], s[4]);
    pos = weno5_left_v<O>(
        weno5_inv<O>(f[1], f[2], f[3], e[1], e[2], e[3], e[4]), s[1], s[2],
        s[3], s[4], s[5]);
  } else if constexpr (SCHEME == 1) {
    typename O::V i0, i1;
    weno3_inv<O>(s[0], s[1], s[2], i0, i1);
    neg = weno3_side_v<O>(i0, i1, s[0], s[1], s[2], true);
    weno3_inv<O>(s[1], s[2], s[3], i0, i1);
    pos = weno3_side_v<O>(i0, i1, s[1], s[2], s[3], false);
  } else if constexpr (SCHEME == 2) {
    neg = O::fma(O::splat(S(0.5)), muscl_slope_v<O>(s[0], s[1], s[2], limiter), s[1]);
    pos = O::fma(O::splat(S(-0.5)), muscl_slope_v<O>(s[1], s[2], s[3], limiter), s[2]);
  } else {
    neg = s[0];
    pos = s[0];
  }
}

// Both faces of cell c from s[k] = v[c-CL+k] (CellStencil<SCHEME>): `left`
// is the pos value of face c-1/2, `right` the neg value of face c+1/2, bit
// for bit what recon_face gives for them.
template <int SCHEME, class O>
__device__ __forceinline__ void recon_cell(const typename O::V* s, int limiter,
                                           typename O::V& left,
                                           typename O::V& right) {
  using S = typename O::S;
  if constexpr (SCHEME == 0) {
    typename O::V e[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) e[k] = O::sub(s[k + 1], s[k]);
    const Weno5Inv<O> w = weno5_inv<O>(
        weno5_tri<O>(e[0], e[1]), weno5_tri<O>(e[1], e[2]),
        weno5_tri<O>(e[2], e[3]), e[0], e[1], e[2], e[3]);
    right = weno5_right_v<O>(w, s[0], s[1], s[2], s[3], s[4]);
    left = weno5_left_v<O>(w, s[0], s[1], s[2], s[3], s[4]);
  } else if constexpr (SCHEME == 1) {
    typename O::V i0, i1;
    weno3_inv<O>(s[0], s[1], s[2], i0, i1);
    right = weno3_side_v<O>(i0, i1, s[0], s[1], s[2], true);
    left = weno3_side_v<O>(i0, i1, s[0], s[1], s[2], false);
  } else if constexpr (SCHEME == 2) {
    const typename O::V sl = muscl_slope_v<O>(s[0], s[1], s[2], limiter);
    right = O::fma(O::splat(S(0.5)), sl, s[1]);
    left = O::fma(O::splat(S(-0.5)), sl, s[1]);
  } else {
    left = s[0];
    right = s[1];
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
    const T gb[3][3], T h_d, T rh_d, T nu, T inv_pr, T* f) {
  // Backward differences along D of u, v, w and T = p/(rho R); rh_d = 1/h_d.
  T bd[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) bd[c] = divk(ub[c] - ua[c], h_d, rh_d);
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
  T q = -(T(0.5) * (ka + kb)) * divk(tb - ta, h_d, rh_d);
  T dot = uf[0] * tau[0] + uf[1] * tau[1] + uf[2] * tau[2];
#pragma unroll
  for (int c = 0; c < 3; ++c) f[1 + c] = f[1 + c] + (-tau[c]);
  f[4] = f[4] + (q + (-dot));
}

}  // namespace swc
