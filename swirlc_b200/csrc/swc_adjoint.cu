// Reverse mode (vector-Jacobian product) of one fused RK stage for WENO5 or
// MUSCL with HLL or HLLC (+ viscous) on a halo-filled state: the discrete
// adjoint used to differentiate whole runs (gradients with respect to the
// initial state and to the kinematic viscosity nu). For a stage
// out = A*u0 + B*(uk + dt*L(uk)) the caller needs
// lambda_out^T dout/duk = B*lambda + B*dt*H^T J_L^T lambda,
// where H is the halo fill; swc_rk_stage_vjp computes
//   vout = beta * H^T J_L(H uk)^T lambda   (beta = B*dt),
//   nu_bar += beta * lambda . dL/dnu.
//
// L(u)_c = S_c - sum_d (F_d[c+1/2] - F_d[c-1/2]) / h_d, so the cotangent of a
// face flux is Fbar = beta * (lambda_right - lambda_left) / h_d. Each face is
// recomputed forward (reconstruction, Riemann flux, viscous flux) and then
// reversed by hand; the reverse of every piece follows the forward code in
// swc_physics.cuh line by line. Primitive cotangents (rho, u, v, w, e, p, h)
// are gathered per cell first and turned into conserved cotangents once per
// cell (the reverse of cons_to_prim), then the halo fill is reversed dim by
// dim in the order z, y, x.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdint.h>
#include <string.h>

#include "swc_launch.h"
#include "swirlc_b200.h"

namespace swc {
namespace {

// ---------------------------------------------------------------------------
// Reverse of the pieces of one face flux.
// ---------------------------------------------------------------------------

// Reverse of recon_cell<0, O> (swc_physics.cuh) on one or two variables
// (the lanes of O): both WENO5 face values of the cell v[2] from
// v[0..4] = v[c-2 .. c+2], which share the smoothness indicators.
// vb[k] += d right/dv[k] * rb + d left/dv[k] * lb. Per stencil r:
// a_r = sum A[r][k] v[k], b_r = sum Bc[r][k] v[k],
// beta_r = 13/12 a_r^2 + 1/4 b_r^2 + eps, candidate q_r = sum Q[r][k] v[k].
template <class O>
__device__ __forceinline__ void weno5_cell_vjp_v(const typename O::V* v,
                                                 typename O::V rb,
                                                 typename O::V lb,
                                                 typename O::V* vb) {
  using S = typename O::S;
  using V = typename O::V;
  constexpr double A[3][5] = {{0, 0, 1, -2, 1}, {0, 1, -2, 1, 0}, {1, -2, 1, 0, 0}};
  constexpr double Bc[3][5] = {{0, 0, 3, -4, 1}, {0, 1, 0, -1, 0}, {1, -4, 3, 0, 0}};
  constexpr double QR[3][5] = {{0, 0, 1.0 / 3, 5.0 / 6, -1.0 / 6},
                               {0, -1.0 / 6, 5.0 / 6, 1.0 / 3, 0},
                               {1.0 / 3, -7.0 / 6, 11.0 / 6, 0, 0}};
  constexpr double QL[3][5] = {{0, 0, 11.0 / 6, -7.0 / 6, 1.0 / 3},
                               {0, 1.0 / 3, 5.0 / 6, -1.0 / 6, 0},
                               {-1.0 / 6, 5.0 / 6, 1.0 / 3, 0, 0}};
  constexpr double DR[3] = {0.3, 0.6, 0.1}, DL[3] = {0.1, 0.6, 0.3};
  // acc + c x with c a nonzero stencil coefficient (c = +-1 as an add).
  auto term = [](double c, V x, V acc, bool first) -> V {
    if (first) return c == 1 ? x : O::mul(O::splat(S(c)), x);
    if (c == 1) return O::add(acc, x);
    if (c == -1) return O::sub(acc, x);
    return O::fma(O::splat(S(c)), x, acc);
  };
  auto lin = [&](const double* c) -> V {
    V acc = O::splat(S(0));
    bool first = true;
#pragma unroll
    for (int k = 0; k < 5; ++k)
      if (c[k] != 0) {
        acc = term(c[k], v[k], acc, first);
        first = false;
      }
    return acc;
  };
  const V c1312 = O::splat(S(13.0 / 12.0)), eps = O::splat(S(1e-6));
  V av[3], bv[3], ib[3], iq[3], qr[3], ql[3];
  V sr, sl, nr, nl;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    av[r] = lin(A[r]);
    bv[r] = lin(Bc[r]);
    qr[r] = lin(QR[r]);
    ql[r] = lin(QL[r]);
    const V be = O::add(O::fma(O::mul(c1312, av[r]), av[r],
                               O::mul(O::mul(O::splat(S(0.25)), bv[r]), bv[r])),
                        eps);
    ib[r] = O::rcp(be);         // 1 / beta_r
    iq[r] = O::mul(ib[r], ib[r]);  // 1 / beta_r^2
    const V ar = O::mul(O::splat(S(DR[r])), iq[r]);
    const V al = O::mul(O::splat(S(DL[r])), iq[r]);
    if (r == 0) {
      sr = ar;
      sl = al;
      nr = O::mul(ar, qr[r]);
      nl = O::mul(al, ql[r]);
    } else {
      sr = O::add(sr, ar);
      sl = O::add(sl, al);
      nr = O::fma(ar, qr[r], nr);
      nl = O::fma(al, ql[r], nl);
    }
  }
  const V isr = O::rcp(sr), isl = O::rcp(sl);
  const V outr = O::mul(nr, isr), outl = O::mul(nl, isl);
  const V gr = O::mul(rb, isr), gl = O::mul(lb, isl);
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    // alpha_r = D_r / beta_r^2; out = sum alpha q / sum alpha.
    const V gdr = O::mul(gr, O::splat(S(DR[r])));
    const V gdl = O::mul(gl, O::splat(S(DL[r])));
    const V qbr = O::mul(gdr, iq[r]);
    const V qbl = O::mul(gdl, iq[r]);
    const V ibq = O::fma(gdr, O::sub(qr[r], outr),
                         O::mul(gdl, O::sub(ql[r], outl)));
    // d(1/beta^2)/d beta = -2 / beta^3
    const V bb = O::mul(O::mul(O::mul(O::splat(S(-2)), ibq), iq[r]), ib[r]);
    const V ca = O::mul(O::mul(bb, O::splat(S(2.0 * 13.0 / 12.0))), av[r]);
    const V cb = O::mul(O::mul(bb, O::splat(S(0.5))), bv[r]);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      if (QR[r][k] != 0) vb[k] = O::fma(O::splat(S(QR[r][k])), qbr, vb[k]);
      if (QL[r][k] != 0) vb[k] = O::fma(O::splat(S(QL[r][k])), qbl, vb[k]);
      if (A[r][k] != 0) vb[k] = term(A[r][k], ca, vb[k], false);
      if (Bc[r][k] != 0) vb[k] = term(Bc[r][k], cb, vb[k], false);
    }
  }
}

// Primitive cotangents of one face state, rotated frame (u[0] normal).
template <typename T>
struct PrimBar {
  T r, u[3], e, p, h;
  __device__ __forceinline__ void zero() {
    r = e = p = h = T(0);
    u[0] = u[1] = u[2] = T(0);
  }
};

// d sqrt(x) = dx / (2 sqrt(x)), zero where the root is zero.
template <typename T>
__device__ __forceinline__ T dsqrt(T root, T bar) {
  return root > T(0) ? bar / (T(2) * root) : T(0);
}

// Forward values of hll_speeds<T, 0> that its reverse needs.
template <typename T>
struct SpeedsFwd {
  T cl, cr, rl, rr, inv, nu_[3], ru[3], nh, rc, s_l, s_r;
  bool lmin_a, rmax_a;  // which candidate min / max picked
};
template <typename T>
__device__ __forceinline__ SpeedsFwd<T> speeds_fwd(const Prim<T>& l,
                                                   const Prim<T>& r, T pe) {
  const T gam = K<T>::gamma(), gm1 = K<T>::gm1();
  SpeedsFwd<T> w;
  w.cl = sqrt_(gam * l.p / l.r);
  w.cr = sqrt_(gam * r.p / r.r);
  w.rl = sqrt_(l.r);
  w.rr = sqrt_(r.r);
  const T den = w.rl + w.rr;
  w.inv = den == T(0) ? T(0) : T(1) / den;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    w.nu_[i] = w.rl * l.u[i] + w.rr * r.u[i];
    w.ru[i] = w.nu_[i] * w.inv;
  }
  w.nh = w.rl * l.h + w.rr * r.h;
  const T rh = w.nh * w.inv;
  const T hs = rh - T(0.5) * (w.ru[0] * w.ru[0] + w.ru[1] * w.ru[1] +
                              w.ru[2] * w.ru[2]) - pe;
  w.rc = sqrt_(gm1 * hs);
  const T sla = l.u[0] - w.cl, slb = w.ru[0] - w.rc;
  const T sra = r.u[0] + w.cr, srb = w.ru[0] + w.rc;
  w.lmin_a = sla <= slb;
  w.rmax_a = sra >= srb;
  w.s_l = w.lmin_a ? sla : slb;
  w.s_r = w.rmax_a ? sra : srb;
  return w;
}

// Reverse of speeds_fwd for the cotangents slb_ of s_l and srb_ of s_r.
template <typename T>
__device__ __forceinline__ void speeds_vjp(const SpeedsFwd<T>& w,
                                           const Prim<T>& l, const Prim<T>& r,
                                           T slb_, T srb_, PrimBar<T>& lb,
                                           PrimBar<T>& rb) {
  const T gam = K<T>::gamma(), gm1 = K<T>::gm1();
  T clb = T(0), crb = T(0), rcb = T(0), rub[3] = {T(0), T(0), T(0)};
  if (w.lmin_a) {
    lb.u[0] += slb_;
    clb += -slb_;
  } else {
    rub[0] += slb_;
    rcb += -slb_;
  }
  if (w.rmax_a) {
    rb.u[0] += srb_;
    crb += srb_;
  } else {
    rub[0] += srb_;
    rcb += srb_;
  }
  const T hsb = dsqrt(w.rc, rcb) * gm1;
  const T rhb = hsb;
#pragma unroll
  for (int i = 0; i < 3; ++i) rub[i] += -hsb * w.ru[i];
  T rlb = T(0), rrb = T(0), invb = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    rlb += rub[i] * l.u[i] * w.inv;
    lb.u[i] += rub[i] * w.rl * w.inv;
    rrb += rub[i] * r.u[i] * w.inv;
    rb.u[i] += rub[i] * w.rr * w.inv;
    invb += rub[i] * w.nu_[i];
  }
  rlb += rhb * l.h * w.inv;
  lb.h += rhb * w.rl * w.inv;
  rrb += rhb * r.h * w.inv;
  rb.h += rhb * w.rr * w.inv;
  invb += rhb * w.nh;
  const T denb = -invb * w.inv * w.inv;
  rlb += denb;
  rrb += denb;
  lb.r += dsqrt(w.rl, rlb);
  rb.r += dsqrt(w.rr, rrb);
  // c = sqrt(gamma p / rho)
  const T cl2b = dsqrt(w.cl, clb), cr2b = dsqrt(w.cr, crb);
  lb.p += cl2b * gam / l.r;
  lb.r += -cl2b * gam * l.p / (l.r * l.r);
  rb.p += cr2b * gam / r.r;
  rb.r += -cr2b * gam * r.p / (r.r * r.r);
}

// Reverse of physical_flux<T, 0>(q, q.p) for the flux cotangent gb.
template <typename T>
__device__ __forceinline__ void phys_vjp(const Prim<T>& q, const T* gb,
                                         PrimBar<T>& qb) {
  const T m = q.r * q.u[0];
  const T eh = q.e + q.p / q.r;
  const T mb = gb[0] + gb[1] * q.u[0] + gb[2] * q.u[1] + gb[3] * q.u[2] +
               gb[4] * eh;
  qb.u[0] += gb[1] * m;
  qb.u[1] += gb[2] * m;
  qb.u[2] += gb[3] * m;
  qb.p += gb[1] + gb[4] * m / q.r;
  qb.e += gb[4] * m;
  qb.r += -gb[4] * m * q.p / (q.r * q.r);
  qb.r += mb * q.u[0];
  qb.u[0] += mb * q.r;
}

// Reverse of hllc_flux<T, 0> with p_dyn = p (no helper states): fb is the
// cotangent of the 5 flux components (rotated momentum order).
template <typename T>
__device__ __forceinline__ void hllc_vjp(const Prim<T>& l, const Prim<T>& r,
                                         T pe, const T* fb, PrimBar<T>& lb,
                                         PrimBar<T>& rb) {
  // ---- forward
  const SpeedsFwd<T> w = speeds_fwd(l, r, pe);
  const T s_l = w.s_l, s_r = w.s_r;
  const T vl = l.u[0], vr = r.u[0];
  const T num = (r.p - l.p) + l.r * vl * (s_l - vl) - r.r * vr * (s_r - vr);
  const T dd = l.r * (s_l - vl) - r.r * (s_r - vr);
  T s_m = dd == T(0) ? T(0) : num / dd;
  const bool clamp = abs_(s_m) < T(1e-6) || dd == T(0);
  if (abs_(s_m) < T(1e-6)) s_m = T(0);
  const bool c1 = s_l >= T(0);
  const bool c2 = (s_l <= T(0)) && (s_m >= T(0));
  const bool c3 = (s_m <= T(0)) && (s_r >= T(0));
  const bool left = c1 || c2;
  const bool star = !c1 && (c2 || c3);
  const Prim<T>& q = left ? l : r;
  PrimBar<T>& qb = left ? lb : rb;
  const T s_k = left ? s_l : s_r;
  // ---- reverse: physical flux of side k
  phys_vjp(q, fb, qb);
  T skb = T(0), smb = T(0);
  if (star) {
    const T v = q.u[0];
    const T g = s_k - s_m;
    const T rat = g == T(0) ? T(0) : s_k / g;
    const T tt = g == T(0) ? T(0) : (s_k - v) / g;
    const T dv = s_m - v;
    T ratb = T(0), dvb = T(0), vb = T(0), ttb = T(0);
    // f0 += rho dv rat
    qb.r += fb[0] * dv * rat;
    dvb += fb[0] * q.r * rat;
    ratb += fb[0] * q.r * dv;
    // f1 += rho s_k (tt s_m - v)
    qb.r += fb[1] * s_k * (tt * s_m - v);
    skb += fb[1] * q.r * (tt * s_m - v);
    ttb += fb[1] * q.r * s_k * s_m;
    smb += fb[1] * q.r * s_k * tt;
    vb += -fb[1] * q.r * s_k;
    // f2, f3 += rho dv u_i rat
#pragma unroll
    for (int i = 1; i < 3; ++i) {
      const T f = fb[1 + i];
      qb.r += f * dv * q.u[i] * rat;
      dvb += f * q.r * q.u[i] * rat;
      qb.u[i] += f * q.r * dv * rat;
      ratb += f * q.r * dv * q.u[i];
    }
    // f4 += rho rat dv W, W = e + p/rho + (s_k - v) s_m
    const T W = q.e + q.p / q.r + (s_k - v) * s_m;
    qb.r += fb[4] * rat * dv * W;
    ratb += fb[4] * q.r * dv * W;
    dvb += fb[4] * q.r * rat * W;
    const T Wb = fb[4] * q.r * rat * dv;
    qb.e += Wb;
    qb.p += Wb / q.r;
    qb.r += -Wb * q.p / (q.r * q.r);
    skb += Wb * s_m;
    vb += -Wb * s_m;
    smb += Wb * (s_k - v);
    // dv = s_m - v
    smb += dvb;
    vb += -dvb;
    if (g != T(0)) {
      // rat = s_k / g, tt = (s_k - v) / g, g = s_k - s_m
      const T ig = T(1) / g;
      skb += ratb * (ig - s_k * ig * ig) + ttb * (ig - (s_k - v) * ig * ig);
      smb += ratb * s_k * ig * ig + ttb * (s_k - v) * ig * ig;
      vb += -ttb * ig;
    }
    qb.u[0] += vb;
  }
  // ---- wave speeds
  T slb_ = left ? skb : T(0), srb_ = left ? T(0) : skb;
  if (!clamp) {
    const T numb = smb / dd;
    const T ddb = -smb * num / (dd * dd);
    lb.p -= numb;
    rb.p += numb;
    lb.r += numb * vl * (s_l - vl) + ddb * (s_l - vl);
    lb.u[0] += numb * l.r * (s_l - T(2) * vl) - ddb * l.r;
    slb_ += numb * l.r * vl + ddb * l.r;
    rb.r += -numb * vr * (s_r - vr) - ddb * (s_r - vr);
    rb.u[0] += -numb * r.r * (s_r - T(2) * vr) + ddb * r.r;
    srb_ += -numb * r.r * vr - ddb * r.r;
  }
  speeds_vjp(w, l, r, slb_, srb_, lb, rb);
}

// sign(x) with sign(0) = 0: the derivative of |x| on the branch taken.
template <typename T>
__device__ __forceinline__ T sgn0(T x) {
  return x > T(0) ? T(1) : (x < T(0) ? T(-1) : T(0));
}

// Reverse of hll_flux<T, 0> with p_dyn = p (no helper states):
// F = t1 F_R + t2 F_L - t3 (U_R - U_L) with t1 = dnn(min(s_r, 0) -
// min(s_l, 0), s_r - s_l), t2 = 1 - t1, t3 = dnn(s_r |s_l| - s_l |s_r|,
// 2 (s_r - s_l)) (hll.py:107-170); fb as in hllc_vjp.
template <typename T>
__device__ __forceinline__ void hll_vjp(const Prim<T>& l, const Prim<T>& r,
                                        T pe, const T* fb, PrimBar<T>& lb,
                                        PrimBar<T>& rb) {
  // ---- forward
  const SpeedsFwd<T> w = speeds_fwd(l, r, pe);
  const T s_l = w.s_l, s_r = w.s_r;
  const T ds = s_r - s_l;
  const T A = min_(s_r, T(0)) - min_(s_l, T(0));
  const T B = s_r * abs_(s_l) - s_l * abs_(s_r);
  const T t1 = ds == T(0) ? T(0) : A / ds;
  const T t3 = ds == T(0) ? T(0) : B / (T(2) * ds);
  const T t2 = T(1) - t1;
  const T m_l = l.r * l.u[0], m_r = r.r * r.u[0];
  const T fl[5] = {m_l, m_l * l.u[0] + l.p, m_l * l.u[1], m_l * l.u[2],
                   m_l * (l.e + l.p / l.r)};
  const T fr[5] = {m_r, m_r * r.u[0] + r.p, m_r * r.u[1], m_r * r.u[2],
                   m_r * (r.e + r.p / r.r)};
  const T ul[5] = {l.r, l.r * l.u[0], l.r * l.u[1], l.r * l.u[2], l.r * l.e};
  const T ur[5] = {r.r, r.r * r.u[0], r.r * r.u[1], r.r * r.u[2], r.r * r.e};
  // ---- reverse
  T t1b = T(0), t3b = T(0), flb[5], frb[5], db[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    t1b += fb[k] * (fr[k] - fl[k]);  // t2 = 1 - t1
    t3b -= fb[k] * (ur[k] - ul[k]);
    frb[k] = fb[k] * t1;
    flb[k] = fb[k] * t2;
    db[k] = -fb[k] * t3;  // cotangent of U_R - U_L
  }
  phys_vjp(l, flb, lb);
  phys_vjp(r, frb, rb);
  // U = (rho, rho u, rho e)
  auto cons_vjp = [](const Prim<T>& q, T sgn, const T* ub, PrimBar<T>& qb) {
    qb.r += sgn * (ub[0] + ub[1] * q.u[0] + ub[2] * q.u[1] + ub[3] * q.u[2] +
                   ub[4] * q.e);
#pragma unroll
    for (int i = 0; i < 3; ++i) qb.u[i] += sgn * ub[1 + i] * q.r;
    qb.e += sgn * ub[4] * q.r;
  };
  cons_vjp(r, T(1), db, rb);
  cons_vjp(l, T(-1), db, lb);
  T slb_ = T(0), srb_ = T(0);
  if (ds != T(0)) {
    const T Ab = t1b / ds, Bb = t3b / (T(2) * ds);
    const T dsb = -(t1b * A) / (ds * ds) - (t3b * B) / (T(2) * ds * ds);
    if (s_r < T(0)) srb_ += Ab;
    if (s_l < T(0)) slb_ -= Ab;
    srb_ += Bb * (abs_(s_l) - s_l * sgn0(s_r));
    slb_ += Bb * (s_r * sgn0(s_l) - abs_(s_r));
    srb_ += dsb;
    slb_ -= dsb;
  }
  speeds_vjp(w, l, r, slb_, srb_, lb, rb);
}

// Reverse of muscl_slope (limiters 1-3) and of muscl_slope_v's van Leer
// slope (0): adds sb * d slope / d(vm1, v0, vp1) to bm1, b0, bp1, on the
// branch the forward takes.
template <typename T>
__device__ __forceinline__ void muscl_slope_vjp(T vm1, T v0, T vp1,
                                                int limiter, T sb, T& bm1,
                                                T& b0, T& bp1) {
  const T dp = vp1 - v0, dm = v0 - vm1;
  T gdm = T(0), gdp = T(0);  // d slope / d dm, d slope / d dp
  if (limiter == 0) {
    // 2 dm dp / (dm + dp) where dm dp > 0, else 0.
    if (dm * dp > T(0)) {
      const T is = T(1) / (dm + dp);
      gdm = T(2) * dp * dp * is * is;
      gdp = T(2) * dm * dm * is * is;
    }
  } else if (limiter == 3) {
    // Smallest magnitude of c2 = (vp1 - vm1) / 4, dp and dm where all
    // three share a sign.
    const T c2 = (vp1 - vm1) * T(0.25);
    const bool up = c2 > T(0) && dp > T(0) && dm > T(0);
    const bool down = c2 < T(0) && dp < T(0) && dm < T(0);
    if (up || down) {
      const T ac = abs_(c2), ap = abs_(dp), am = abs_(dm);
      if (ac <= ap && ac <= am) {
        bp1 += T(0.25) * sb;
        bm1 -= T(0.25) * sb;
        return;
      }
      if (ap <= am) gdp = T(1);
      else gdm = T(1);
    }
  } else if (dp != T(0)) {
    // phi(r) dp with r = dm / dp: d/d dm = phi'(r), d/d dp = phi - phi' r.
    const T r = dm / dp;
    T m, dmr;
    if (limiter == 1) {  // max(0, min(min(2 r, (1 + r) / 2), 2))
      const T a = T(2) * r, b = T(0.5) * (T(1) + r);
      m = a <= b ? a : b;
      dmr = a <= b ? T(2) : T(0.5);
      if (!(m <= T(2))) {
        m = T(2);
        dmr = T(0);
      }
    } else {  // minmod: max(0, min(r, 1))
      m = r <= T(1) ? r : T(1);
      dmr = r <= T(1) ? T(1) : T(0);
    }
    const T phi = m > T(0) ? m : T(0);
    const T dphi = m > T(0) ? dmr : T(0);
    gdm = dphi;
    gdp = phi - dphi * r;
  }
  // dp = vp1 - v0, dm = v0 - vm1. (dp = 0 gives r = 0 and phi(0) = 0 for
  // both ratio limiters, so the slope and its derivative vanish there.)
  bp1 += sb * gdp;
  b0 += sb * (gdm - gdp);
  bm1 -= sb * gdm;
}

// Reverse of recon_cell<2> (MUSCL) on one lane: right = v0 + slope / 2,
// left = v0 - slope / 2 with cotangents rb, lb.
template <typename T>
__device__ __forceinline__ void muscl_cell_vjp(T vm1, T v0, T vp1, T rb, T lb,
                                               int limiter, T& bm1, T& b0,
                                               T& bp1) {
  b0 += rb + lb;
  muscl_slope_vjp(vm1, v0, vp1, limiter, T(0.5) * (rb - lb), bm1, b0, bp1);
}
__device__ __forceinline__ void muscl_cell_vjp(float2 vm1, float2 v0,
                                               float2 vp1, float2 rb,
                                               float2 lb, int limiter,
                                               float2& bm1, float2& b0,
                                               float2& bp1) {
  muscl_cell_vjp(vm1.x, v0.x, vp1.x, rb.x, lb.x, limiter, bm1.x, b0.x, bp1.x);
  muscl_cell_vjp(vm1.y, v0.y, vp1.y, rb.y, lb.y, limiter, bm1.y, b0.y, bp1.y);
}
__device__ __forceinline__ void muscl_cell_vjp(double2 vm1, double2 v0,
                                               double2 vp1, double2 rb,
                                               double2 lb, int limiter,
                                               double2& bm1, double2& b0,
                                               double2& bp1) {
  muscl_cell_vjp(vm1.x, v0.x, vp1.x, rb.x, lb.x, limiter, bm1.x, b0.x, bp1.x);
  muscl_cell_vjp(vm1.y, v0.y, vp1.y, rb.y, lb.y, limiter, bm1.y, b0.y, bp1.y);
}

// Both face values of the cell v[2] from the five cells v[0..4] =
// v[c-2 .. c+2] of the face kernel's window (MUSCL uses v[1..3]).
template <int SCHEME, class O>
__device__ __forceinline__ void recon5(const typename O::V* v, int limiter,
                                       typename O::V& left,
                                       typename O::V& right) {
  if constexpr (SCHEME == 0) recon_cell<0, O>(v, limiter, left, right);
  else recon_cell<2, O>(v + 1, limiter, left, right);
}
// Reverse of recon5: vb[k] += d right / dv[k] * rb + d left / dv[k] * lb.
template <int SCHEME, class O>
__device__ __forceinline__ void cell_vjp5(const typename O::V* v,
                                          typename O::V rb, typename O::V lb,
                                          int limiter, typename O::V* vb) {
  if constexpr (SCHEME == 0) weno5_cell_vjp_v<O>(v, rb, lb, vb);
  else muscl_cell_vjp(v[1], v[2], v[3], rb, lb, limiter, vb[1], vb[2], vb[3]);
}

// Reverse of the Riemann flux RIEMANN (0 HLL, 1 HLLC).
template <int RIEMANN, typename T>
__device__ __forceinline__ void riemann_vjp(const Prim<T>& l,
                                            const Prim<T>& r, T pe,
                                            const T* fb, PrimBar<T>& lb,
                                            PrimBar<T>& rb) {
  if constexpr (RIEMANN == 0) hll_vjp<T>(l, r, pe, fb, lb, rb);
  else hllc_vjp<T>(l, r, pe, fb, lb, rb);
}

// Reverse of viscous_flux<T, 0> for the cotangent fb[1..4]. gab/gbb are the
// cotangents of the tangential central differences ga[1][1], ga[1][0],
// ga[2][2], ga[2][0] (and the same for b). Returns fb . F_visc / nu, the
// viscous part's derivative with respect to nu (the flux is linear in nu).
template <typename T>
__device__ __forceinline__ T viscous_vjp(T ra, T rb, const T* ua, const T* ub,
                                         T pa, T pb, const T* ga4,
                                         const T* gb4, T h, T nu, T inv_pr,
                                         const T* fb, T& rab, T& rbb, T* uab,
                                         T* ubb, T& pab, T& pbb, T* gab,
                                         T* gbb) {
  const T R = K<T>::r_gas(), cp = K<T>::cp();
  // forward (ga4/gb4 = g11, g10, g22, g20)
  T bd[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) bd[c] = (ub[c] - ua[c]) / h;
  const T g0 = bd[0], g1 = T(0.5) * (ga4[0] + gb4[0]),
          g2 = T(0.5) * (ga4[2] + gb4[2]);
  const T div = g0 + g1 + g2;
  const T rf = T(0.5) * (ra + rb);
  T s[3];
  s[0] = bd[0] - T(1.0 / 3.0) * div;
  s[1] = T(0.5) * (bd[1] + T(0.5) * (ga4[1] + gb4[1]));
  s[2] = T(0.5) * (bd[2] + T(0.5) * (ga4[3] + gb4[3]));
  T tau[3], uf[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    tau[c] = T(2) * rf * nu * s[c];
    uf[c] = T(0.5) * (ua[c] + ub[c]);
  }
  const T ta = pa / (ra * R), tb = pb / (rb * R);
  const T ka = inv_pr * cp * (nu * ra), kb = inv_pr * cp * (nu * rb);
  const T kf = T(0.5) * (ka + kb);
  const T q = -kf * ((tb - ta) / h);
  const T dot = uf[0] * tau[0] + uf[1] * tau[1] + uf[2] * tau[2];
  const T dnu = -(fb[1] * tau[0] + fb[2] * tau[1] + fb[3] * tau[2]) +
                fb[4] * (q - dot);
  // reverse
  T taub[3], sb[3], bdb[3] = {T(0), T(0), T(0)};
  T rfb = T(0);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    taub[c] = -fb[1 + c] - fb[4] * uf[c];
    const T ufb = -fb[4] * tau[c];
    uab[c] += T(0.5) * ufb;
    ubb[c] += T(0.5) * ufb;
    rfb += taub[c] * T(2) * nu * s[c];
    sb[c] = taub[c] * T(2) * rf * nu;
  }
  const T qb = fb[4];
  const T kfb = -qb * ((tb - ta) / h);
  const T tbb = -qb * kf / h, tab = qb * kf / h;
  rab += T(0.5) * kfb * inv_pr * cp * nu;
  rbb += T(0.5) * kfb * inv_pr * cp * nu;
  pab += tab / (ra * R);
  rab += -tab * pa / (ra * ra * R);
  pbb += tbb / (rb * R);
  rbb += -tbb * pb / (rb * rb * R);
  rab += T(0.5) * rfb;
  rbb += T(0.5) * rfb;
  const T divb = -sb[0] * T(1.0 / 3.0);
  bdb[0] += sb[0] + divb;
  bdb[1] += T(0.5) * sb[1];
  bdb[2] += T(0.5) * sb[2];
  gab[1] += T(0.25) * sb[1];
  gbb[1] += T(0.25) * sb[1];
  gab[3] += T(0.25) * sb[2];
  gbb[3] += T(0.25) * sb[2];
  gab[0] += T(0.5) * divb;
  gbb[0] += T(0.5) * divb;
  gab[2] += T(0.5) * divb;
  gbb[2] += T(0.5) * divb;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    ubb[c] += bdb[c] / h;
    uab[c] -= bdb[c] / h;
  }
  return nu > T(0) ? dnu / nu : T(0);
}

// ---------------------------------------------------------------------------
// Kernels.
// ---------------------------------------------------------------------------
struct VjpArgs {
  int nx, ny, nz, h;
  long long sx, sz;
  double dx, dy, dz;
  const void* uk[5];
  const void* lam[5];
  void* prim[7];  // rho, u, v, w, e, p, h of uk, every cell
  void* pbar[7];  // primitive cotangents of the x and z faces, every cell
  // Copies in the layout [z][y][x] (x contiguous) for the y faces, whose
  // lines run along the contiguous axis of the reference layout: the
  // primitives, lam, and the y faces' primitive cotangents.
  void* primT[7];
  void* lamT[5];
  void* pbarT[7];
  long long tsy, tsz;  // y and z strides of the transposed layout
  void* vout[5];  // conserved cotangents, every cell
  const void* pe[3];
  int has_pe;
  int visc;
  double nu, pr;
  double beta;
  int gravity_mask;
  double g[3];
  double* nu_bar;
  int seg;  // faces per thread along a line
  int limiter;  // MUSCL limiter (SWC_LIM_*)
  // vout = alpha*lam + c1*x1 + c2*x2 + beta*H^T J^T lam on the interior.
  double alpha, c1, c2;
  const void* x1[5];
  const void* x2[5];
  // Per face pass D (in that pass's layout), so that every sum has a fixed
  // order: primitive cotangents of the five cells at the head of each
  // segment (hb), the cotangents of each cell's four tangential differences
  // (tg; tgh: the head cell's part from its segment's first face), and the
  // nu cotangent of every block (nu_part, pass D from nu_off[D]).
  // vjp_fix_kernel adds the first two to the primitive cotangents.
  void* hb[3][7];
  void* tg[3][4];
  void* tgh[3][4];
  double* nu_part;
  long long nu_off[3];
};

template <typename T>
__device__ __forceinline__ T pe_of(const VjpArgs& a, int xa, int ya, int za) {
  if (!a.has_pe) return T(0);
  const T* px = static_cast<const T*>(a.pe[0]);
  const T* py = static_cast<const T*>(a.pe[1]);
  const T* pz = static_cast<const T*>(a.pe[2]);
  return (-(px ? px[xa] : T(0)) - (py ? py[ya] : T(0))) - (pz ? pz[za] : T(0));
}

// Tiles of the prim and cell kernels: a (32, 8) block covers 32 x 32 (y, x)
// cells of one z plane, 4 per thread; the transposed copies go through a
// shared-memory tile so that both layouts are read and written coalesced.
constexpr int TT = 32;
// Faces per thread of a face pass. The five head cells of consecutive
// segments must not overlap (vjp_fix_kernel adds each once).
constexpr int kVjpSeg = 16;
static_assert(kVjpSeg >= 5, "segment heads would overlap");

// Primitives of every cell (halos included), in both layouts, with their
// cotangent buffers cleared, and lam transposed.
// Dynamic shared memory of the transposing kernels: one [TT][TT+1] tile
// per transposed variable, so a single barrier separates all writers from
// all readers.
constexpr int kPrimTiles = 12;  // 7 primitives + 5 lambda fields
constexpr int kCellTiles = 7;   // 7 primitive cotangents
template <typename T>
__device__ __forceinline__ T (*vjp_tiles())[TT][TT + 1] {
  extern __shared__ __align__(16) unsigned char vjp_smem[];
  return reinterpret_cast<T(*)[TT][TT + 1]>(vjp_smem);
}

template <typename T>
__global__ void __launch_bounds__(256) vjp_prim_kernel(const VjpArgs a) {
  T(*tiles)[TT][TT + 1] = vjp_tiles<T>();
  const int nxa = a.nx + 2 * a.h, nya = a.ny + 2 * a.h;
  const int za = blockIdx.z;
  const int y0 = blockIdx.x * TT, x0 = blockIdx.y * TT;
  const int tx = threadIdx.x, ty = threadIdx.y;
  // All loads first (the stores go to arrays the compiler cannot tell apart
  // from the loaded ones), then the primitives.
  T cv[4][5], lv[4][5];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int xa = x0 + ty + 8 * k, ya = y0 + tx;
    const bool in = xa < nxa && ya < nya;
    const long long o = za * a.sz + xa * a.sx + ya;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      cv[k][v] = in ? static_cast<const T*>(a.uk[v])[o] : T(1);
      lv[k][v] = in ? static_cast<const T*>(a.lam[v])[o] : T(0);
    }
  }
  T pr[4][7];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int xa = x0 + ty + 8 * k, ya = y0 + tx;
    T u, vv, w, e, p, hh;
    cons_to_prim(cv[k][0], cv[k][1], cv[k][2], cv[k][3], cv[k][4],
                 pe_of<T>(a, min(xa, nxa - 1), min(ya, nya - 1), za), u, vv,
                 w, e, p, hh);
    pr[k][0] = cv[k][0]; pr[k][1] = u; pr[k][2] = vv; pr[k][3] = w;
    pr[k][4] = e; pr[k][5] = p; pr[k][6] = hh;
    if (xa >= nxa || ya >= nya) continue;
    const long long o = za * a.sz + xa * a.sx + ya;
#pragma unroll
    for (int v = 0; v < 7; ++v) {
      static_cast<T*>(a.prim[v])[o] = pr[k][v];
      static_cast<T*>(a.pbar[v])[o] = T(0);
    }
  }
  // tiles[v][x - x0][y - y0]; the transposed write reads them along x.
#pragma unroll
  for (int v = 0; v < kPrimTiles; ++v) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      tiles[v][ty + 8 * k][tx] = v < 7 ? pr[k][v] : lv[k][v - 7];
  }
  __syncthreads();
#pragma unroll
  for (int v = 0; v < kPrimTiles; ++v) {
    T(*tile)[TT + 1] = tiles[v];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int yl = ty + 8 * k;
      const int xa = x0 + tx, ya = y0 + yl;
      if (xa >= nxa || ya >= nya) continue;
      const long long ot = za * a.tsz + ya * a.tsy + xa;
      if (v < 7) {
        static_cast<T*>(a.primT[v])[ot] = tile[tx][yl];
        static_cast<T*>(a.pbarT[v])[ot] = T(0);
      } else {
        static_cast<T*>(a.lamT[v - 7])[ot] = tile[tx][yl];
      }
    }
  }
}

// Face VJPs along dim D. Thread = `seg` consecutive faces of one line along
// D; a register window holds the 6-cell stencil primitives and their
// cotangents, and a cell's cotangents are added to pbar once, when the
// window leaves it. Neighbouring threads take neighbouring lines along the
// contiguous axis: y for the x and z faces in the reference layout, x for
// the y faces, which run on the transposed copies.
// Minimum resident blocks of the face kernel (its register budget).
#ifndef SWC_VJP_FACE_MINB
#define SWC_VJP_FACE_MINB 1
#endif

template <typename T, int D, int SCHEME, int RIEMANN>
__global__ void __launch_bounds__(128, SWC_VJP_FACE_MINB)
    vjp_face_kernel(const VjpArgs a) {
  const int h = a.h;
  const int n = D == 0 ? a.nx : (D == 1 ? a.ny : a.nz);
  // Transverse axes (t1, t2) of the rotated frame: x:(y,z) y:(x,z) z:(x,y).
  const int n1 = D == 0 ? a.ny : a.nx;
  const int n2 = D == 2 ? a.ny : a.nz;
  const long long st = D == 0 ? a.sx : (D == 1 ? a.tsy : a.sz);
  const long long s1 = D == 2 ? a.sx : 1;
  const long long s2 = D == 0 ? a.sz : (D == 1 ? a.tsz : 1);
  void* const* PBAR = D == 1 ? a.pbarT : a.pbar;
  const void* const* LAM = D == 1 ? const_cast<const void* const*>(a.lamT)
                                  : a.lam;
  const T hd = T(D == 0 ? a.dx : (D == 1 ? a.dy : a.dz));
  const T h1 = T(D == 0 ? a.dy : a.dx);
  const T h2 = T(D == 2 ? a.dy : a.dz);
  const int nseg = (n + 1 + a.seg - 1) / a.seg;
  // Thread index: the transverse coordinate along the contiguous axis
  // varies fastest (coalesced loads and atomics).
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long lines = (long long)n1 * n2;
  // Threads past the last line take no faces but join the nu reduction.
  const bool active = tid < lines * nseg;
  int c1, c2, sg;
  {
    long long r = tid;
    if (D == 2) {  // (t1, t2) = (x, y): y fastest
      c2 = (int)(r % n2); r /= n2;
      c1 = (int)(r % n1); r /= n1;
    } else {  // t1: y for D = 0; x (contiguous when transposed) for D = 1
      c1 = (int)(r % n1); r /= n1;
      c2 = (int)(r % n2); r /= n2;
    }
    sg = (int)r;
  }
  const int i0 = active ? sg * a.seg : 0;
  const int i1 = active ? min(i0 + a.seg, n + 1) : 0;
  const long long base = (long long)(c1 + h) * s1 + (long long)(c2 + h) * s2;
  const int vel[3] = {1 + D, D == 0 ? 2 : 1, D == 2 ? 2 : 3};
  const T* P[7];
#pragma unroll
  for (int k = 0; k < 7; ++k)
    P[k] = static_cast<const T*>(D == 1 ? a.primT[k] : a.prim[k]);
  // The 7 rotated primitives (rho, u_n, u_t1, u_t2, e, p, h) are held as
  // the pairs (rho, e), (u_n, u_t1), (u_t2, p) and h alone, the grouping of
  // the forward stage's reconstruction: each pair is one two-lane
  // instruction stream (Two<T>), h a one-lane one (One<T>).
  using O2 = Two<T>;
  using O1 = One<T>;
  using V2 = typename O2::V;
  // Rotated primitives of cell j (normal index with halo = j + h).
  auto load = [&](int j, V2* q, T& qh) {
    const long long o = base + (long long)(j + h) * st;
    q[0] = O2::mk(P[0][o], P[4][o]);
    q[1] = O2::mk(P[vel[0]][o], P[vel[1]][o]);
    q[2] = O2::mk(P[vel[2]][o], P[5][o]);
    qh = P[6][o];
  };
  auto lam_at = [&](int j, T* lv) {
    if (j < 0 || j >= n) {
#pragma unroll
      for (int v = 0; v < 5; ++v) lv[v] = T(0);
      return;
    }
    const long long o = base + (long long)(j + h) * st;
#pragma unroll
    for (int v = 0; v < 5; ++v) lv[v] = static_cast<const T*>(LAM[v])[o];
  };
  // A thread flushes cells i0-3 .. i1+1 of its line, each once. The five
  // head cells i0-3 .. i0+1 are also flushed by the previous segment's
  // thread (they are its tail): this thread's part goes to hb, which the
  // fix-up kernel adds. Every other cell gets exactly one addition in this
  // pass, so the atomic below adds to a value no other thread changes
  // meanwhile and the sum is the same on every run.
  auto flush = [&](int j, const V2* b, T bh) {
    const long long o = base + (long long)(j + h) * st;
    const T val[7] = {b[0].x, b[1].x, b[1].y, b[2].x, b[0].y, b[2].y, bh};
    const int var[7] = {0, vel[0], vel[1], vel[2], 4, 5, 6};
    if (j <= i0 + 1) {
#pragma unroll
      for (int k = 0; k < 7; ++k) static_cast<T*>(a.hb[D][var[k]])[o] = val[k];
    } else {
#pragma unroll
      for (int k = 0; k < 7; ++k) atomicAdd(static_cast<T*>(PBAR[var[k]]) + o, val[k]);
    }
  };
  // Window at face i (between cells i-1 and i): primitives sw[k] of cells
  // i-3+k (k = 0..5) and cotangents ab[k] of cells i-3+k (k = 0..4). Step i
  // reconstructs cell i (its left value is face i's right state; its right
  // value is carried to face i+1), reverses face i's flux, and then reverses
  // cell i-1's reconstruction with the cotangents of both of its face values
  // (face i-1's, carried, and face i's). A cell whose two faces belong to two
  // threads is reversed by both, each with its own face's cotangent (the
  // reverse is linear in them). Cells leave the window complete.
  V2 sw[6][3], ab[5][3];
  T swh[6], abh[5];
  const V2 z2 = O2::splat(T(0));
#pragma unroll
  for (int k = 0; k < 5; ++k) {
#pragma unroll
    for (int v = 0; v < 3; ++v) ab[k][v] = z2;
    abh[k] = T(0);
  }
  // Right value of cell i-1; cotangent of its left value.
  V2 qn[3] = {z2, z2, z2}, cl[3] = {z2, z2, z2};
  T qnh = T(0), clh = T(0);
  T la[5], lb[5];
  if (active) {
#pragma unroll
    for (int k = 0; k < 5; ++k) load(i0 - 3 + k, sw[k], swh[k]);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const V2 s5[5] = {sw[0][v], sw[1][v], sw[2][v], sw[3][v], sw[4][v]};
      V2 lv;
      recon5<SCHEME, O2>(s5, a.limiter, lv, qn[v]);
    }
    const T s5[5] = {swh[0], swh[1], swh[2], swh[3], swh[4]};
    T lv;
    recon5<SCHEME, O1>(s5, a.limiter, lv, qnh);
  }
  lam_at(active ? i0 - 1 : -1, la);
  const T scale = T(a.beta) / hd;
  const T nu = T(a.nu), inv_pr = T(1.0 / a.pr);
  const T i2t1 = T(1) / (T(2) * h1), i2t2 = T(1) / (T(2) * h2);
  // Viscous: tangential central differences of cell o (g11, g10, g22, g20:
  // velocity t1 and the normal velocity along t1, velocity t2 and the normal
  // velocity along t2). Their cotangents are stored per cell (tg; the head
  // cell i0-1 of a segment, whose face i0-1 belongs to the previous
  // segment, into tgh) and moved onto the four neighbours by the fix-up
  // kernel, which gathers them per target cell in a fixed order.
  auto tang = [&](long long o, T* g4) {
    g4[0] = (P[vel[1]][o + s1] - P[vel[1]][o - s1]) * i2t1;
    g4[1] = (P[vel[0]][o + s1] - P[vel[0]][o - s1]) * i2t1;
    g4[2] = (P[vel[2]][o + s2] - P[vel[2]][o - s2]) * i2t2;
    g4[3] = (P[vel[0]][o + s2] - P[vel[0]][o - s2]) * i2t2;
  };
  auto tang_store = [&](long long o, const T* gb, bool head) {
    void* const* dst = head ? a.tgh[D] : a.tg[D];
#pragma unroll
    for (int c = 0; c < 4; ++c) static_cast<T*>(dst[c])[o] = gb[c];
  };
  // Tangential differences of cell i-1 and their cotangent so far.
  T g4a[4] = {T(0), T(0), T(0), T(0)}, gba[4] = {T(0), T(0), T(0), T(0)};
  if (a.visc && active) tang(base + (long long)(i0 - 1 + h) * st, g4a);
  T nub = T(0);
  for (int i = i0; i < i1; ++i) {
    load(i + 2, sw[5], swh[5]);
    if (i + 1 < i1) {
      // Start the next step's global reads (window cell i+3, lambda of cell
      // i+1, tangential neighbours of cell i+1) towards L1: the flux
      // reverse of this step hides their latency.
      const long long o3 = base + (long long)(i + 3 + h) * st;
      prefetch_l1(P[0] + o3);
      prefetch_l1(P[4] + o3);
      prefetch_l1(P[5] + o3);
      prefetch_l1(P[6] + o3);
#pragma unroll
      for (int k = 0; k < 3; ++k) prefetch_l1(P[vel[k]] + o3);
      const long long o1 = base + (long long)(i + 1 + h) * st;
      if (i + 1 < n) {
#pragma unroll
        for (int v = 0; v < 5; ++v) prefetch_l1(static_cast<const T*>(LAM[v]) + o1);
      }
      if (a.visc) {
        prefetch_l1(P[vel[1]] + o1 + s1);
        prefetch_l1(P[vel[1]] + o1 - s1);
        prefetch_l1(P[vel[0]] + o1 + s1);
        prefetch_l1(P[vel[0]] + o1 - s1);
        prefetch_l1(P[vel[2]] + o1 + s2);
        prefetch_l1(P[vel[2]] + o1 - s2);
        prefetch_l1(P[vel[0]] + o1 + s2);
        prefetch_l1(P[vel[0]] + o1 - s2);
      }
    }
    lam_at(i, lb);
    T fb[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) fb[v] = (lb[v] - la[v]) * scale;
    // Rotate the flux cotangent to the rotated momentum order.
    T fr[5];
    fr[0] = fb[0];
    fr[1] = fb[1 + D];
    fr[2] = fb[1 + (D == 0 ? 1 : 0)];
    fr[3] = fb[1 + (D == 2 ? 1 : 2)];
    fr[4] = fb[4];
    // Forward: cell i from cells i-2 .. i+2; face i's states.
    V2 lv[3], rn[3];
    T lvh, rnh;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const V2 s5[5] = {sw[1][v], sw[2][v], sw[3][v], sw[4][v], sw[5][v]};
      recon5<SCHEME, O2>(s5, a.limiter, lv[v], rn[v]);
    }
    {
      const T s5[5] = {swh[1], swh[2], swh[3], swh[4], swh[5]};
      recon5<SCHEME, O1>(s5, a.limiter, lvh, rnh);
    }
    Prim<T> ql, qr;
    ql.r = qn[0].x; ql.u[0] = qn[1].x; ql.u[1] = qn[1].y; ql.u[2] = qn[2].x;
    ql.e = qn[0].y; ql.p = qn[2].y; ql.h = qnh;
    qr.r = lv[0].x; qr.u[0] = lv[1].x; qr.u[1] = lv[1].y; qr.u[2] = lv[2].x;
    qr.e = lv[0].y; qr.p = lv[2].y; qr.h = lvh;
    int xa, ya, za;  // face cell b = i (pe at the face index)
    {
      const int jb = i + h;
      if (D == 0) { xa = jb; ya = c1 + h; za = c2 + h; }
      else if (D == 1) { ya = jb; xa = c1 + h; za = c2 + h; }
      else { za = jb; xa = c1 + h; ya = c2 + h; }
    }
    const T pe = pe_of<T>(a, xa, ya, za);
    PrimBar<T> lbar, rbar;
    lbar.zero();
    rbar.zero();
    riemann_vjp<RIEMANN, T>(ql, qr, pe, fr, lbar, rbar);
    if (a.visc) {
      // Cells a = i-1 (window 2) and b = i (window 3).
      // Cell a: rho, u, p (rotated frame) from the pairs.
      const T ra_ = sw[2][0].x, rb_ = sw[3][0].x;
      const T pa_ = sw[2][2].y, pb_ = sw[3][2].y;
      const long long ob = base + (long long)(i + h) * st;
      T g4b[4];
      tang(ob, g4b);
      T rab = T(0), rbb = T(0), pab = T(0), pbb = T(0);
      T uab[3] = {T(0), T(0), T(0)}, ubb[3] = {T(0), T(0), T(0)};
      T gab[4] = {T(0), T(0), T(0), T(0)}, gbb[4] = {T(0), T(0), T(0), T(0)};
      const T ua[3] = {sw[2][1].x, sw[2][1].y, sw[2][2].x};
      const T ub[3] = {sw[3][1].x, sw[3][1].y, sw[3][2].x};
      nub += viscous_vjp<T>(ra_, rb_, ua, ub, pa_, pb_, g4a, g4b, hd, nu,
                            inv_pr, fr, rab, rbb, uab, ubb, pab, pbb, gab, gbb);
      ab[2][0].x += rab;
      ab[3][0].x += rbb;
      ab[2][2].y += pab;
      ab[3][2].y += pbb;
      ab[2][1].x += uab[0];
      ab[3][1].x += ubb[0];
      ab[2][1].y += uab[1];
      ab[3][1].y += ubb[1];
      ab[2][2].x += uab[2];
      ab[3][2].x += ubb[2];
      // Cell i-1's tangential cotangent is complete (faces i-1 and i),
      // except at i = i0 (face i0 only: the head part).
#pragma unroll
      for (int c = 0; c < 4; ++c) gba[c] += gab[c];
      tang_store(ob - st, gba, i == i0);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        gba[c] = gbb[c];
        g4a[c] = g4b[c];
      }
    }
    // Reverse of cell i-1's reconstruction (cells i-3 .. i+1).
    {
      const V2 cr[3] = {O2::mk(lbar.r, lbar.e), O2::mk(lbar.u[0], lbar.u[1]),
                        O2::mk(lbar.u[2], lbar.p)};
#pragma unroll
      for (int v = 0; v < 3; ++v) {
        const V2 s5[5] = {sw[0][v], sw[1][v], sw[2][v], sw[3][v], sw[4][v]};
        V2 acc[5] = {ab[0][v], ab[1][v], ab[2][v], ab[3][v], ab[4][v]};
        cell_vjp5<SCHEME, O2>(s5, cr[v], cl[v], a.limiter, acc);
#pragma unroll
        for (int k = 0; k < 5; ++k) ab[k][v] = acc[k];
      }
      {
        const T s5[5] = {swh[0], swh[1], swh[2], swh[3], swh[4]};
        T acc[5] = {abh[0], abh[1], abh[2], abh[3], abh[4]};
        cell_vjp5<SCHEME, O1>(s5, lbar.h, clh, a.limiter, acc);
#pragma unroll
        for (int k = 0; k < 5; ++k) abh[k] = acc[k];
      }
      cl[0] = O2::mk(rbar.r, rbar.e);
      cl[1] = O2::mk(rbar.u[0], rbar.u[1]);
      cl[2] = O2::mk(rbar.u[2], rbar.p);
      clh = rbar.h;
#pragma unroll
      for (int v = 0; v < 3; ++v) qn[v] = rn[v];
      qnh = rnh;
    }
    // Cell i-3 is complete: flush it and slide.
    flush(i - 3, ab[0], abh[0]);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
#pragma unroll
      for (int v = 0; v < 3; ++v) sw[k][v] = sw[k + 1][v];
      swh[k] = swh[k + 1];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
      for (int v = 0; v < 3; ++v) ab[k][v] = ab[k + 1][v];
      abh[k] = abh[k + 1];
    }
#pragma unroll
    for (int v = 0; v < 3; ++v) ab[4][v] = z2;
    abh[4] = T(0);
#pragma unroll
    for (int v = 0; v < 5; ++v) la[v] = lb[v];
  }
  if (active) {
    // Cell i1-1: only its left face (face i1-1) belongs to this thread.
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const V2 s5[5] = {sw[0][v], sw[1][v], sw[2][v], sw[3][v], sw[4][v]};
      V2 acc[5] = {ab[0][v], ab[1][v], ab[2][v], ab[3][v], ab[4][v]};
      cell_vjp5<SCHEME, O2>(s5, z2, cl[v], a.limiter, acc);
#pragma unroll
      for (int k = 0; k < 5; ++k) ab[k][v] = acc[k];
    }
    {
      const T s5[5] = {swh[0], swh[1], swh[2], swh[3], swh[4]};
      T acc[5] = {abh[0], abh[1], abh[2], abh[3], abh[4]};
      cell_vjp5<SCHEME, O1>(s5, T(0), clh, a.limiter, acc);
#pragma unroll
      for (int k = 0; k < 5; ++k) abh[k] = acc[k];
    }
    // Cells i1-3 .. i1+1 may still hold contributions.
#pragma unroll
    for (int k = 0; k < 5; ++k) flush(i1 - 3 + k, ab[k], abh[k]);
    // Cell i1-1: its face i1-1 part (face i1 is the next segment's).
    if (a.visc) tang_store(base + (long long)(i1 - 1 + h) * st, gba, false);
  }
  if (a.visc && a.nu_bar) {
    // One partial per block (a fixed shuffle tree per warp, the warps in
    // order), summed in a fixed order by vjp_nu_kernel.
    __shared__ double wsum[32];
    double m = double(nub);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      m += __shfl_xor_sync(0xffffffffu, m, off);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += wsum[w];
      a.nu_part[a.nu_off[D] + blockIdx.x] = b;
    }
  }
}

// The parts of face pass D that the pass leaves outside pbar / pbarT, for
// the target cell (c1, c2, j) of that pass's frame (interior indices; o its
// offset in the pass's layout), added to acc (7 primitive cotangents): the
// head parts of the segments (hb) and, viscous, the tangential-difference
// cotangents of the four neighbouring source cells (tg, plus tgh where the
// source is the head cell i0-1 of a segment), always in the same order.
// vjp_fix_kernel calls it once per pass for each cell, so no two threads
// write one sum and the result does not depend on scheduling.
template <typename T, int D>
__device__ __forceinline__ int pass_parts(const VjpArgs& a, int c1, int c2,
                                          int j, long long o, T* acc) {
  const int n = D == 0 ? a.nx : (D == 1 ? a.ny : a.nz);
  const int n1 = D == 0 ? a.ny : a.nx;
  const int n2 = D == 2 ? a.ny : a.nz;
  const long long s1 = D == 2 ? a.sx : 1;
  const long long s2 = D == 0 ? a.sz : (D == 1 ? a.tsz : 1);
  constexpr int seg = kVjpSeg;  // a.seg
  const int nseg = (n + 1 + seg - 1) / seg;
  const bool in1 = c1 >= 0 && c1 < n1, in2 = c2 >= 0 && c2 < n2;
  const int vel[3] = {1 + D, D == 0 ? 2 : 1, D == 2 ? 2 : 3};
  int mask = 0;
  // Head cells of segment sg: sg*seg-3 .. sg*seg+1 (seg >= 5: disjoint).
  if (in1 && in2 && j >= -3 && (j + 3) % seg <= 4 && (j + 3) / seg < nseg) {
#pragma unroll
    for (int v = 0; v < 7; ++v) acc[v] += static_cast<const T*>(a.hb[D][v])[o];
    mask = 0x7f;
  }
  if (!a.visc || j < -1 || j > n || !(in1 || in2) || c1 < -1 || c1 > n1 ||
      c2 < -1 || c2 > n2)
    return mask;
  // Cotangent k of the tangential differences of source cell
  // (j, c1+d1, c2+d2): its tg value (cells 0 .. n of a line) plus its tgh
  // value where it is the head cell i0-1 of a segment.
  const bool hj = (j + 1) % seg == 0 && (j + 1) / seg < nseg;
  auto src = [&](int k, int d1, int d2) -> T {
    const int e1 = c1 + d1, e2 = c2 + d2;
    if (e1 < 0 || e1 >= n1 || e2 < 0 || e2 >= n2) return T(0);
    const long long q = o + d1 * s1 + d2 * s2;
    T v = j >= 0 ? static_cast<const T*>(a.tg[D][k])[q] : T(0);
    if (hj) v += static_cast<const T*>(a.tgh[D][k])[q];
    return v;
  };
  const T h1 = T(D == 0 ? a.dy : a.dx);
  const T h2 = T(D == 2 ? a.dy : a.dz);
  const T i2t1 = T(1) / (T(2) * h1), i2t2 = T(1) / (T(2) * h2);
  // A source adds +g/(2 h_t) to its upper and -g/(2 h_t) to its lower
  // neighbour along t.
  acc[vel[1]] += (src(0, -1, 0) - src(0, 1, 0)) * i2t1;
  acc[vel[0]] += (src(1, -1, 0) - src(1, 1, 0)) * i2t1 +
                 (src(3, 0, -1) - src(3, 0, 1)) * i2t2;
  acc[vel[2]] += (src(2, 0, -1) - src(2, 0, 1)) * i2t2;
  return mask | (1 << vel[0]) | (1 << vel[1]) | (1 << vel[2]);
}

// The face passes' parts outside pbar / pbarT (pass_parts), one thread per
// cell of the padded grid: L = 0 adds the x and z passes' parts to pbar
// (reference layout), L = 1 the y pass's to pbarT (transposed layout). No
// two threads write one cell.
template <typename T, int L>
__global__ void __launch_bounds__(256) vjp_fix_kernel(const VjpArgs a) {
  const int h = a.h;
  const unsigned nxa = a.nx + 2 * h, nya = a.ny + 2 * h, nza = a.nz + 2 * h;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nxa * nya * nza) return;
  // 32-bit division: the host keeps the padded grid below 2^32 cells.
  const unsigned tt = (unsigned)t;
  T acc[7] = {T(0), T(0), T(0), T(0), T(0), T(0), T(0)};
  int mask;
  long long o;
  void* const* PB;
  if (L == 0) {  // (y fastest, x, z)
    const unsigned q = tt / nya;
    const int ya = (int)(tt - q * nya);
    const int za = (int)(q / nxa);
    const int xa = (int)(q - (unsigned)za * nxa);
    o = za * a.sz + xa * a.sx + ya;
    mask = pass_parts<T, 0>(a, ya - h, za - h, xa - h, o, acc);
    mask |= pass_parts<T, 2>(a, xa - h, ya - h, za - h, o, acc);
    PB = a.pbar;
  } else {  // transposed: (x fastest, y, z)
    const unsigned q = tt / nxa;
    const int xt = (int)(tt - q * nxa);
    const int za = (int)(q / nya);
    const int yt = (int)(q - (unsigned)za * nya);
    o = za * a.tsz + yt * a.tsy + xt;
    mask = pass_parts<T, 1>(a, xt - h, za - h, yt - h, o, acc);
    PB = a.pbarT;
  }
  if (!mask) return;
  // Every load before any store (the compiler cannot tell PB from the
  // arrays read above, and a load after a store would wait for it).
  T cur[7];
#pragma unroll
  for (int v = 0; v < 7; ++v)
    cur[v] = (mask >> v) & 1 ? static_cast<const T*>(PB[v])[o] : T(0);
#pragma unroll
  for (int v = 0; v < 7; ++v)
    if ((mask >> v) & 1) static_cast<T*>(PB[v])[o] = cur[v] + acc[v];
}

// nu_bar += the per-warp partials of the three face passes, summed in a
// fixed order by one block.
__global__ void __launch_bounds__(256) vjp_nu_kernel(const double* part,
                                                     long long count,
                                                     double* nu_bar) {
  __shared__ double red[256];
  double m = 0.0;
  for (long long i = threadIdx.x; i < count; i += 256) m += part[i];
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *nu_bar += red[0];
}

// Conserved cotangents of every cell from its primitive cotangents (the
// reverse of cons_to_prim), plus the gravity source rho*G*g. The y faces'
// cotangents are read back from the transposed layout through a tile.
// Two resident blocks per SM in single precision (128 registers, 8 bytes
// spilled: 1.7 % off the checkpointed KH 128^3 sweep, same gradient bits);
// double precision needs ~250 registers and keeps one.
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) vjp_cell_kernel(const VjpArgs a) {
  T(*tiles)[TT][TT + 1] = vjp_tiles<T>();  // as in vjp_prim_kernel
  const int nxa = a.nx + 2 * a.h, nya = a.ny + 2 * a.h;
  const int za = blockIdx.z;
  const int y0 = blockIdx.x * TT, x0 = blockIdx.y * TT;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const T gm1 = K<T>::gm1();
  // Loads first (see vjp_prim_kernel): the cotangents of both layouts and
  // the state, then the y faces' cotangents through the tile, then lam and
  // the caller's terms.
  T pbs[4][7], pbt[4][7], c4[4][5];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int xa = x0 + ty + 8 * k, ya = y0 + tx;
    const bool in = xa < nxa && ya < nya;
    const long long o = za * a.sz + xa * a.sx + ya;
    const int xt = x0 + tx, yt = y0 + ty + 8 * k;
    const bool int_ = xt < nxa && yt < nya;
    const long long ot = za * a.tsz + yt * a.tsy + xt;
#pragma unroll
    for (int v = 0; v < 7; ++v) {
      pbs[k][v] = in ? static_cast<const T*>(a.pbar[v])[o] : T(0);
      pbt[k][v] = int_ ? static_cast<const T*>(a.pbarT[v])[ot] : T(0);
    }
#pragma unroll
    for (int v = 0; v < 5; ++v)
      c4[k][v] = in ? static_cast<const T*>(a.uk[v])[o] : T(1);
  }
  // tiles[v][y - y0][x - x0], written along x, read along y.
#pragma unroll
  for (int v = 0; v < kCellTiles; ++v) {
#pragma unroll
    for (int k = 0; k < 4; ++k) tiles[v][ty + 8 * k][tx] = pbt[k][v];
  }
  __syncthreads();
#pragma unroll
  for (int v = 0; v < kCellTiles; ++v) {
#pragma unroll
    for (int k = 0; k < 4; ++k) pbs[k][v] += tiles[v][tx][ty + 8 * k];
  }
  T l4[4][5], x14[4][5], x24[4][5];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int xa = x0 + ty + 8 * k, ya = y0 + tx;
    const bool in = xa < nxa && ya < nya;
    const long long o = za * a.sz + xa * a.sx + ya;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      l4[k][v] = in ? static_cast<const T*>(a.lam[v])[o] : T(0);
      x14[k][v] = in && a.x1[v] ? static_cast<const T*>(a.x1[v])[o] : T(0);
      x24[k][v] = in && a.x2[v] ? static_cast<const T*>(a.x2[v])[o] : T(0);
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int xa = x0 + ty + 8 * k, ya = y0 + tx;
    if (xa >= nxa || ya >= nya) continue;
    const long long o = za * a.sz + xa * a.sx + ya;
    const T* c = c4[k];
    const T* pb = pbs[k];
    const T pe = pe_of<T>(a, xa, ya, za);
    const T rho = c[0];
    const T inv = T(1) / rho;
    const T u[3] = {inv * c[1], inv * c[2], inv * c[3]};
    const T e = inv * c[4];
    const T eint = e - T(0.5) * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) - pe;
    const T p = gm1 * rho * eint;
    // h = e + p / rho
    T eb = pb[4] + pb[6];
    T pbb = pb[5] + pb[6] / rho;
    T rb = pb[0] - pb[6] * p / (rho * rho);
    // p = gm1 rho eint
    rb += pbb * gm1 * eint;
    const T eintb = pbb * gm1 * rho;
    // eint = e - |u|^2/2 - pe
    eb += eintb;
    T ub[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) ub[i] = pb[1 + i] - eintb * u[i];
    // e = inv E, u_i = inv m_i
    T invb = eb * c[4];
    T out[5];
    out[4] = eb * inv;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      out[1 + i] = ub[i] * inv;
      invb += ub[i] * c[1 + i];
    }
    rb += -invb * inv * inv;
    // Gravity source on the momenta of interior cells.
    const bool interior = xa >= a.h && xa < a.nx + a.h && ya >= a.h &&
                          ya < a.ny + a.h && za >= a.h && za < a.nz + a.h;
    if (a.gravity_mask && interior) {
#pragma unroll
      for (int d = 0; d < 3; ++d)
        if (a.gravity_mask & (1 << d))
          rb += T(a.beta) * l4[k][1 + d] * K<T>::grav() * T(a.g[d]);
    }
    out[0] = rb;
    // The caller's combination on the interior (alpha*lam + c1*x1 + c2*x2):
    // added before the halo reverse, which is linear and moves only halo
    // cotangents.
    if (interior) {
#pragma unroll
      for (int v = 0; v < 5; ++v)
        out[v] += T(a.alpha) * l4[k][v] + T(a.c1) * x14[k][v] +
                  T(a.c2) * x24[k][v];
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) static_cast<T*>(a.vout[v])[o] = out[v];
  }
}

// Reverse of the halo fill (swc_halo_fill: x, then y, then z) on vout.
// Each forward pass writes the halo layers of one dim over the whole padded
// plane of the other two, so the fill is H = H_z H_y H_x and its reverse
// applies H_z^T, H_y^T, H_x^T in turn: one launch per dim, one thread per
// (field, column along that dim). A thread reads its column's halo cells,
// clears them and adds each cotangent to the cell it was copied from (the
// wrapped cell, periodic; the edge cell, Neumann; none, Dirichlet or
// unfilled). Each column belongs to one thread and its additions come in a
// fixed order, so the sums do not depend on scheduling.
struct VjpHalo {
  int nx, ny, nz, h;
  long long sx, sz;
  void* f[5];
  int kind[5][3][2];  // fill kind per field, dim and side
};

template <typename T>
__global__ void __launch_bounds__(256) vjp_halo_kernel(const VjpHalo a,
                                                       const int d) {
  const int h = a.h;
  // Plane axes (a, b) of the column's dim d: (x, y) for z, (z, x) for y,
  // (z, y) for x, the contiguous axis y fastest where it is in the plane.
  const int nxa = a.nx + 2 * h, nya = a.ny + 2 * h, nza = a.nz + 2 * h;
  const int na = d == 2 ? nxa : nza;
  const int nb = d == 1 ? nxa : nya;
  const long long sa = d == 2 ? a.sx : a.sz;
  const long long sb = d == 1 ? a.sx : 1;
  const long long sd = d == 0 ? a.sx : (d == 1 ? 1 : a.sz);
  const int n = d == 0 ? a.nx : (d == 1 ? a.ny : a.nz);
  const unsigned plane = (unsigned)na * (unsigned)nb;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 5LL * plane) return;
  const unsigned tt = (unsigned)t;
  const int v = (int)(tt / plane);
  const unsigned pp = tt - (unsigned)v * plane;
  const int ia = (int)(pp / (unsigned)nb);
  const int ib = (int)(pp - (unsigned)ia * (unsigned)nb);
  T* f = static_cast<T*>(a.f[v]) + ia * sa + ib * sb;
  const int kl = a.kind[v][d][0], kh = a.kind[v][d][1];
  const bool per = kl == SWC_BC_PERIODIC;  // then kh is too
  if (h <= 8 && (!per || n >= 2 * h)) {
    // Every value is read before any is written (the compiler cannot tell
    // the cells apart, and a load after a store would wait for it). With
    // n >= 2h the wrapped sources [n, n+h) and [h, 2h) are distinct.
    T lo[8], hi[8], slo[8], shi[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k >= h) break;
      lo[k] = f[k * sd];
      hi[k] = f[(n + h + k) * sd];
      if (per) {
        slo[k] = f[(n + k) * sd];   // source of low halo cell k
        shi[k] = f[(h + k) * sd];   // source of high halo cell k
      }
    }
    T elo = T(0), ehi = T(0);
    if (kl == SWC_BC_NEUMANN || kh == SWC_BC_NEUMANN) {
      elo = f[h * sd];
      ehi = f[(n + h - 1) * sd];
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k >= h) break;
      f[k * sd] = T(0);
      f[(n + h + k) * sd] = T(0);
    }
    if (per) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (k >= h) break;
        f[(n + k) * sd] = slo[k] + lo[k];
        f[(h + k) * sd] = shi[k] + hi[k];
      }
      return;
    }
    // Neumann sides: every halo layer of the side is a copy of its edge
    // cell (n = 1 makes both edge cells one cell: added in turn).
    T sl = T(0), sh = T(0);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (k >= h) break;
      sl += lo[k];
      sh += hi[k];
    }
    if (kl == SWC_BC_NEUMANN && kh == SWC_BC_NEUMANN && n == 1) {
      f[h * sd] = (elo + sl) + sh;
    } else {
      if (kl == SWC_BC_NEUMANN) f[h * sd] = elo + sl;
      if (kh == SWC_BC_NEUMANN) f[(n + h - 1) * sd] = ehi + sh;
    }
    return;
  }
  // General widths, or a periodic dim shorter than 2h (wrapped sources
  // shared by both sides): one cell at a time, in the same order.
  for (int k = 0; k < h; ++k) {
    const T lv = f[k * sd], hv = f[(n + h + k) * sd];
    f[k * sd] = T(0);
    f[(n + h + k) * sd] = T(0);
    if (per) {
      f[(n + k) * sd] += lv;
      f[(h + k) * sd] += hv;
    } else {
      if (kl == SWC_BC_NEUMANN) f[h * sd] += lv;
      if (kh == SWC_BC_NEUMANN) f[(n + h - 1) * sd] += hv;
    }
  }
}

// Above 48 KB of dynamic shared memory a kernel must opt in: done on the
// first call per dtype (whatever the scheme), which the header asks callers
// to make outside stream capture.
template <typename T>
int vjp_smem_opt_in() {
  static bool smem_set = false;
  if (smem_set) return SWC_OK;
  const size_t tile_bytes = sizeof(T) * TT * (TT + 1);
  if (cudaFuncSetAttribute(vjp_prim_kernel<T>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(kPrimTiles * tile_bytes)) != cudaSuccess ||
      cudaFuncSetAttribute(vjp_cell_kernel<T>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(kCellTiles * tile_bytes)) != cudaSuccess)
    return record_error(SWC_ERR_LAUNCH, "stage vjp: shared memory opt-in");
  smem_set = true;
  return SWC_OK;
}

template <typename T, int SCHEME, int RIEMANN>
int launch_vjp(const VjpArgs& a, const SwcFieldBC* bcs, cudaStream_t s) {
  const int nxa = a.nx + 2 * a.h, nya = a.ny + 2 * a.h, nza = a.nz + 2 * a.h;
  const dim3 tgrid((nya + TT - 1) / TT, (nxa + TT - 1) / TT, nza);
  const dim3 tblock(TT, 8);
  const size_t tile_bytes = sizeof(T) * TT * (TT + 1);
  const int st = vjp_smem_opt_in<T>();
  if (st) return st;
  vjp_prim_kernel<T><<<tgrid, tblock, kPrimTiles * tile_bytes, s>>>(a);
  note_launch();
  // Face passes; the blocks' nu partials of pass D start at nu_off[D].
  const int ft = 128;
  VjpArgs b = a;
  unsigned blocks[3];
  long long parts = 0;
  for (int D = 0; D < 3; ++D) {
    const int n = D == 0 ? a.nx : (D == 1 ? a.ny : a.nz);
    const int n1 = D == 0 ? a.ny : a.nx;
    const int n2 = D == 2 ? a.ny : a.nz;
    const long long nseg = (n + 1 + a.seg - 1) / a.seg;
    const long long threads = (long long)n1 * n2 * nseg;
    blocks[D] = (unsigned)((threads + ft - 1) / ft);
    b.nu_off[D] = parts;
    parts += blocks[D];
  }
  for (int D = 0; D < 3; ++D) {
    if (D == 0) vjp_face_kernel<T, 0, SCHEME, RIEMANN><<<blocks[D], ft, 0, s>>>(b);
    else if (D == 1) vjp_face_kernel<T, 1, SCHEME, RIEMANN><<<blocks[D], ft, 0, s>>>(b);
    else vjp_face_kernel<T, 2, SCHEME, RIEMANN><<<blocks[D], ft, 0, s>>>(b);
    note_launch();
  }
  {
    const long long cells = (long long)nxa * nya * nza;
    const unsigned fb = (unsigned)((cells + 255) / 256);
    vjp_fix_kernel<T, 0><<<fb, 256, 0, s>>>(b);
    note_launch();
    vjp_fix_kernel<T, 1><<<fb, 256, 0, s>>>(b);
    note_launch();
  }
  if (b.visc && b.nu_bar) {
    vjp_nu_kernel<<<1, 256, 0, s>>>(b.nu_part, parts, b.nu_bar);
    note_launch();
  }
  vjp_cell_kernel<T><<<tgrid, tblock, kCellTiles * tile_bytes, s>>>(b);
  note_launch();
  {
    VjpHalo hh;
    memset(&hh, 0, sizeof(hh));
    hh.nx = a.nx; hh.ny = a.ny; hh.nz = a.nz; hh.h = a.h;
    hh.sx = a.sx; hh.sz = a.sz;
    for (int v = 0; v < 5; ++v) {
      hh.f[v] = a.vout[v];
      for (int d = 0; d < 3; ++d) {
        int lo = bcs[v].side[d][0].kind, hi = bcs[v].side[d][1].kind;
        if (lo == SWC_BC_PERIODIC || hi == SWC_BC_PERIODIC)
          lo = hi = SWC_BC_PERIODIC;
        hh.kind[v][d][0] = lo;
        hh.kind[v][d][1] = hi;
      }
    }
    // z, then y, then x: the reverse of the fill's order.
    for (int d = 2; d >= 0; --d) {
      const long long cols = 5LL * (d == 0 ? (long long)nya * nza
                                           : (d == 1 ? (long long)nxa * nza
                                                     : (long long)nxa * nya));
      vjp_halo_kernel<T><<<(unsigned)((cols + 255) / 256), 256, 0, s>>>(hh, d);
      note_launch();
    }
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SWC_OK
                          : record_error(SWC_ERR_LAUNCH, "stage vjp: %s",
                                         cudaGetErrorString(e));
}

}  // namespace
}  // namespace swc

namespace swc {
namespace {
int stage_vjp(const SwcGrid* grid, const SwcScheme* sc, const SwcFieldBC* bcs,
              const void* const* uk, const void* const* lam, double alpha,
              double beta, const void* const* x1, double c1,
              const void* const* x2, double c2, void* const* vout,
              double* nu_bar, void* const* scratch, void* stream);
}  // namespace
}  // namespace swc

extern "C" int swc_rk_stage_vjp(const SwcGrid* grid, const SwcScheme* sc,
                                const SwcFieldBC* bcs, const void* const* uk,
                                const void* const* lam, double alpha,
                                double beta, const void* const* x1, double c1,
                                const void* const* x2, double c2,
                                void* const* vout, double* nu_bar,
                                void* const* scratch, void* stream) {
  swc::NvtxRange nvtx_range_("swc_rk_stage_vjp");
  return swc::stage_vjp(grid, sc, bcs, uk, lam, alpha, beta, x1, c1, x2, c2,
                        vout, nu_bar, scratch, stream);
}

// The reversed step: for u' = SSP-RK3(u) (rk3.py:87-120) with stages
//   u1 = u + dt L(u), u2 = 3/4 u + 1/4 (u1 + dt L(u1)),
//   u' = 1/3 u + 2/3 (u2 + dt L(u2)),
// a cotangent g of u' gives g2 = 2/3 g + V(u2, g, 2/3 dt),
// g1 = 1/4 g2 + V(u1, g2, 1/4 dt), gn = 1/3 g + 3/4 g2 + g1 + V(u, g1, dt);
// for RK2 (rk2.py:69-86, u' = 1/2 u + 1/2 (u1 + dt L(u1))):
// g1 = 1/2 g + V(u1, g, 1/2 dt), gn = 1/2 g + g1 + V(u, g1, dt).
extern "C" int swc_rk_step_vjp(const SwcGrid* grid, const SwcScheme* sc,
                               const SwcFieldBC* bcs, int32_t order,
                               const void* const* stages, double dt,
                               const void* const* g, void* const* gn,
                               void* const* work, double* nu_bar,
                               void* const* scratch, void* stream) {
  swc::NvtxRange nvtx_range_("swc_rk_step_vjp");
  using namespace swc;
  if (order != 2 && order != 3)
    return record_error(SWC_ERR_UNSUPPORTED,
                        "Runge-Kutta order %d is not implemented", order);
  if (!stages || !g || !gn || !work)
    return record_error(SWC_ERR_ARG, "step vjp: NULL argument");
  const void* const* u0 = stages;
  const void* const* u1 = stages + 5;
  void* const* w1 = work;      // g1
  void* const* w2 = work + 5;  // g2 (RK3)
  for (int v = 0; v < 5; ++v) {
    for (int k = 0; k < 5 * order; ++k)
      if (gn[v] == stages[k])
        return record_error(SWC_ERR_ARG, "step vjp: gn must not alias a stage");
    for (int k = 0; k < 5; ++k)
      if (gn[v] == g[k])
        return record_error(SWC_ERR_ARG, "step vjp: gn must not alias g");
    for (int k = 0; k < 5 * (order - 1); ++k)
      if (gn[v] == work[k])
        return record_error(SWC_ERR_ARG, "step vjp: gn must not alias work");
  }
  int rc;
  if (order == 3) {
    const void* const* u2 = stages + 10;
    if ((rc = stage_vjp(grid, sc, bcs, u2, g, 2.0 / 3.0, 2.0 / 3.0 * dt,
                        nullptr, 0.0, nullptr, 0.0, w2, nu_bar, scratch,
                        stream)))
      return rc;
    if ((rc = stage_vjp(grid, sc, bcs, u1, w2, 0.25, 0.25 * dt, nullptr, 0.0,
                        nullptr, 0.0, w1, nu_bar, scratch, stream)))
      return rc;
    return stage_vjp(grid, sc, bcs, u0, w1, 1.0, dt, g, 1.0 / 3.0, w2, 0.75,
                     gn, nu_bar, scratch, stream);
  }
  if ((rc = stage_vjp(grid, sc, bcs, u1, g, 0.5, 0.5 * dt, nullptr, 0.0,
                      nullptr, 0.0, w1, nu_bar, scratch, stream)))
    return rc;
  return stage_vjp(grid, sc, bcs, u0, w1, 1.0, dt, g, 0.5, nullptr, 0.0, gn,
                   nu_bar, scratch, stream);
}

namespace swc {
namespace {
int stage_vjp(const SwcGrid* grid, const SwcScheme* sc, const SwcFieldBC* bcs,
              const void* const* uk, const void* const* lam, double alpha,
              double beta, const void* const* x1, double c1,
              const void* const* x2, double c2, void* const* vout,
              double* nu_bar, void* const* scratch, void* stream) {
  int st = check_grid(grid);
  if (st) return st;
  if (!sc || !bcs || !uk || !lam || !vout || !scratch)
    return record_error(SWC_ERR_ARG, "stage vjp: NULL argument");
  if (sc->dtype != SWC_F32 && sc->dtype != SWC_F64)
    return record_error(SWC_ERR_ARG, "bad dtype %d", sc->dtype);
  if ((sc->interp != SWC_WENO5 && sc->interp != SWC_MUSCL) ||
      (sc->riemann != SWC_HLL && sc->riemann != SWC_HLLC) || sc->nscalars != 0)
    return record_error(SWC_ERR_UNSUPPORTED,
                        "the stage adjoint covers WENO5 or MUSCL with HLL or "
                        "HLLC, without transported scalars");
  if (sc->interp == SWC_MUSCL && (sc->limiter < 0 || sc->limiter > 3))
    return record_error(SWC_ERR_ARG, "bad MUSCL limiter %d", sc->limiter);
  if (grid->halo < 3)
    return record_error(SWC_ERR_ARG, "halo_width %d is too small (needs 3)",
                        grid->halo);
  for (int v = 0; v < 5; ++v) {
    if (!uk[v] || !lam[v] || !vout[v])
      return record_error(SWC_ERR_ARG, "stage vjp: NULL field %d", v);
    if (bcs[v].via_primitive)
      return record_error(SWC_ERR_UNSUPPORTED,
                          "the stage adjoint does not cover primitive BCs");
    const int nd[3] = {grid->nx, grid->ny, grid->nz};
    for (int d = 0; d < 3; ++d)
      if ((bcs[v].side[d][0].kind == SWC_BC_PERIODIC ||
           bcs[v].side[d][1].kind == SWC_BC_PERIODIC) &&
          nd[d] < grid->halo)
        return record_error(SWC_ERR_UNSUPPORTED,
                            "stage vjp: periodic dim %d has %d cells, fewer "
                            "than the halo width", d, nd[d]);
  }
  for (int k = 0; k < SWC_VJP_SCRATCH; ++k)
    if (!scratch[k]) return record_error(SWC_ERR_ARG, "NULL scratch field %d", k);
  if (grid->nz + 2 * grid->halo > 65535)
    return record_error(SWC_ERR_ARG, "stage vjp: nz %d is too large", grid->nz);
  VjpArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = grid->nx; a.ny = grid->ny; a.nz = grid->nz; a.h = grid->halo;
  a.sx = grid->sx; a.sz = grid->sz;
  a.dx = grid->dx; a.dy = grid->dy; a.dz = grid->dz;
  for (int v = 0; v < 5; ++v) {
    a.uk[v] = uk[v];
    a.lam[v] = lam[v];
    a.vout[v] = vout[v];
    a.x1[v] = x1 ? x1[v] : nullptr;
    a.x2[v] = x2 ? x2[v] : nullptr;
    if (vout[v] == lam[v] || (x1 && x1[v] == vout[v]) ||
        (x2 && x2[v] == vout[v]) || vout[v] == uk[v])
      return record_error(SWC_ERR_ARG, "stage vjp: vout must not alias its inputs");
  }
  a.alpha = alpha;
  a.c1 = c1;
  a.c2 = c2;
  for (int k = 0; k < 7; ++k) {
    a.prim[k] = scratch[k];
    a.pbar[k] = scratch[7 + k];
    a.primT[k] = scratch[14 + k];
    a.pbarT[k] = scratch[21 + k];
  }
  for (int v = 0; v < 5; ++v) a.lamT[v] = scratch[28 + v];
  for (int D = 0; D < 3; ++D) {
    for (int k = 0; k < 7; ++k) a.hb[D][k] = scratch[33 + 7 * D + k];
    for (int k = 0; k < 4; ++k) {
      a.tg[D][k] = scratch[54 + 4 * D + k];
      a.tgh[D][k] = scratch[66 + 4 * D + k];
    }
  }
  a.nu_part = static_cast<double*>(scratch[78]);
  a.tsy = grid->nx + 2 * grid->halo;
  a.tsz = a.tsy * (long long)(grid->ny + 2 * grid->halo);
  {
    // The per-block nu partials (doubles) live in scratch field 78.
    const long long elems = a.tsz * (long long)(grid->nz + 2 * grid->halo);
    const size_t tsize = sc->dtype == SWC_F32 ? 4 : 8;
    long long parts = 0, most = 0;
    const int nd[3] = {grid->nx, grid->ny, grid->nz};
    for (int D = 0; D < 3; ++D) {
      const long long n1 = nd[D == 0 ? 1 : 0], n2 = nd[D == 2 ? 1 : 2];
      const long long threads = n1 * n2 * ((nd[D] + 1 + kVjpSeg - 1) / kVjpSeg);
      parts += (threads + 127) / 128;
      // Columns of the halo reverse and cells of the fix-up (32-bit index
      // arithmetic).
      most = std::max(most, a.tsz * (long long)(grid->nz + 2 * grid->halo));
      most = std::max(most, 5LL * (n1 + 2LL * grid->halo) *
                                (n2 + 2LL * grid->halo));
    }
    if ((reinterpret_cast<uintptr_t>(scratch[78]) & 7) != 0 ||
        parts * 8 > elems * (long long)tsize)
      return record_error(SWC_ERR_ARG, "stage vjp: scratch field 78 is "
                          "misaligned or too small");
    if (most >= (1LL << 32))
      return record_error(SWC_ERR_ARG, "stage vjp: grid too large");
  }
  for (int d = 0; d < 3; ++d) {
    a.pe[d] = sc->pe_axis[d];
    if (sc->pe_axis[d]) a.has_pe = 1;
    a.g[d] = sc->g[d];
  }
  a.visc = sc->diffusion ? 1 : 0;
  a.nu = sc->nu;
  a.pr = sc->pr > 0 ? sc->pr : 1.0;
  a.beta = beta;
  a.gravity_mask = sc->gravity_mask;
  a.nu_bar = nu_bar;
  a.seg = kVjpSeg;
  a.limiter = sc->limiter;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool f32 = sc->dtype == SWC_F32;
  const bool muscl = sc->interp == SWC_MUSCL, hllc = sc->riemann == SWC_HLLC;
  if (f32) {
    if (muscl) return hllc ? launch_vjp<float, 2, 1>(a, bcs, s)
                           : launch_vjp<float, 2, 0>(a, bcs, s);
    return hllc ? launch_vjp<float, 0, 1>(a, bcs, s)
                : launch_vjp<float, 0, 0>(a, bcs, s);
  }
  if (muscl) return hllc ? launch_vjp<double, 2, 1>(a, bcs, s)
                         : launch_vjp<double, 2, 0>(a, bcs, s);
  return hllc ? launch_vjp<double, 0, 1>(a, bcs, s)
              : launch_vjp<double, 0, 0>(a, bcs, s);
}

}  // namespace
}  // namespace swc
