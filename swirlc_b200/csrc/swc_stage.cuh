// Fused RK stage kernel: halo-filled conserved state -> primitives -> face
// reconstruction -> Riemann (+ viscous) flux -> divergence + source -> stage
// combination, one pass over the grid per RK stage.
//
// Reference path replaced: the rhs of get_rhs_fn
// (compressible_navier_stokes.py:68-268) evaluated inside rk3.integrate /
// rk2.integrate (rk3.py:87-120, rk2.py:69-86).
//
// Work decomposition (2.5-D plane marching). A CTA owns a TY x TX column of
// cells in the (y, x) plane and marches along z over `zseg` planes. A ring
// of RING planes of primitives (with an in-plane halo HR) lives in shared
// memory; each step loads one new plane, computes every y- and x-face of the
// centre plane into shared memory, computes the z-face above each column in
// registers (the face below is carried from the previous step), then forms
// the divergence and the stage update of the centre plane. Each face flux is
// computed exactly once per CTA.
#pragma once

#include "swc_physics.cuh"
#include "swirlc_b200.h"

namespace swc {

struct StageArgs {
  int nx, ny, nz, halo;
  long long sx, sz;
  double dx, dy, dz;
  const void* uk[5];
  const void* u0[5];
  void* uout[5];
  int mode;
  double c0, c1;
  const double* dt;
  double* dtmin_out;
  const void* pe[3];
  int has_pe;
  int limiter;
  double nu, pr;
  int gravity_mask;
  double g[3];
  int zseg;
};

__device__ __forceinline__ void atomic_min_pos(double* addr, double v) {
  // Non-negative doubles order like their bit patterns.
  atomicMin(reinterpret_cast<unsigned long long*>(addr),
            static_cast<unsigned long long>(__double_as_longlong(v)));
}

template <typename T>
__device__ __forceinline__ void set_var(Prim<T>& q, int v, T x) {
  switch (v) {
    case 0: q.r = x; break;
    case 1: q.u[0] = x; break;
    case 2: q.u[1] = x; break;
    case 3: q.u[2] = x; break;
    case 4: q.e = x; break;
    case 5: q.p = x; break;
    default: q.h = x; break;
  }
}

template <int SCHEME, bool VISC>
struct Geom {
  static constexpr int LO = Stencil<SCHEME>::LO;
  static constexpr int RI = Stencil<SCHEME>::RI;
  static constexpr int NW = LO + RI;
  static constexpr int cmax(int a, int b) { return a > b ? a : b; }
  static constexpr int HR = cmax(cmax(LO, RI - 1), VISC ? 1 : 0);
  static constexpr int ZLO = cmax(cmax(LO - 1, VISC ? 1 : 0), 0);
  static constexpr int ZHI = cmax(cmax(RI, VISC ? 1 : 0), 1);
  static constexpr int RING = ZLO + 1 + ZHI;
  // Halo layers the stored arrays need.
  static constexpr int NEED = cmax(HR, cmax(ZLO + 1, ZHI));
};

template <typename T, int SCHEME, bool VISC, int TY, int TX>
struct Layout {
  using G = Geom<SCHEME, VISC>;
  static constexpr int PW = TY + 2 * G::HR;
  static constexpr int PH = TX + 2 * G::HR;
  static constexpr int PS = PW * PH;
  static constexpr int NT = TX * TY;
  static constexpr int RING_ELEMS = G::RING * 7 * PS;
  static constexpr int FY_ELEMS = 5 * TX * (TY + 1);
  static constexpr int FX_ELEMS = 5 * (TX + 1) * TY;
  static constexpr size_t SMEM =
      sizeof(T) * (size_t)(RING_ELEMS + FY_ELEMS + FX_ELEMS);
};

template <typename T, int SCHEME, int RIEMANN, bool VISC, int TY, int TX>
__global__ void __launch_bounds__(TY* TX, sizeof(T) == 4 ? 2 : 1)
    stage_kernel(const StageArgs a) {
  using G = Geom<SCHEME, VISC>;
  using L = Layout<T, SCHEME, VISC, TY, TX>;
  constexpr int LO = G::LO, NW = G::NW, HR = G::HR, ZLO = G::ZLO,
                ZHI = G::ZHI, RING = G::RING;
  constexpr int PW = L::PW, PH = L::PH, PS = L::PS, NT = L::NT;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  T* fy = ring + L::RING_ELEMS;  // [5][TX][TY+1]
  T* fx = fy + L::FY_ELEMS;      // [5][TX+1][TY]

  const int tid = threadIdx.x;
  const int ty = tid % TY, tx = tid / TY;
  const int y0 = blockIdx.x * TY, x0 = blockIdx.y * TX;
  const int z0 = blockIdx.z * a.zseg;
  const int z1 = min(z0 + a.zseg, a.nz);
  const int h = a.halo;
  const int nxa = a.nx + 2 * h, nya = a.ny + 2 * h;
  const long long sx = a.sx, sz = a.sz;

  const T* __restrict__ uk0 = static_cast<const T*>(a.uk[0]);
  const T* __restrict__ uk1 = static_cast<const T*>(a.uk[1]);
  const T* __restrict__ uk2 = static_cast<const T*>(a.uk[2]);
  const T* __restrict__ uk3 = static_cast<const T*>(a.uk[3]);
  const T* __restrict__ uk4 = static_cast<const T*>(a.uk[4]);
  const T* __restrict__ pex = static_cast<const T*>(a.pe[0]);
  const T* __restrict__ pey = static_cast<const T*>(a.pe[1]);
  const T* __restrict__ pez = static_cast<const T*>(a.pe[2]);
  const bool has_pe = a.has_pe != 0;

  const T dx = T(a.dx), dy = T(a.dy), dz = T(a.dz);
  const T nu = T(a.nu), inv_pr = T(1.0 / a.pr);

  auto pe_at = [&](int xa, int ya, int za) -> T {
    if (!has_pe) return T(0);
    T ax = pex ? pex[xa] : T(0);
    T ay = pey ? pey[ya] : T(0);
    T az = pez ? pez[za] : T(0);
    return (-ax - ay) - az;
  };
  auto R = [&](int slot, int v, int px, int py) -> T& {
    return ring[((slot * 7 + v) * PH + px) * PW + py];
  };
  auto load_plane = [&](int z, int slot) {
    const int za = z + h;
    for (int idx = tid; idx < PS; idx += NT) {
      int px = idx / PW, py = idx - px * PW;
      int xa = x0 - HR + px + h, ya = y0 - HR + py + h;
      T r = T(1), ru = T(0), rv = T(0), rw = T(0), re = T(1), pe = T(0);
      if (xa < nxa && ya < nya) {
        long long o = za * sz + xa * sx + ya;
        r = __ldg(uk0 + o);
        ru = __ldg(uk1 + o);
        rv = __ldg(uk2 + o);
        rw = __ldg(uk3 + o);
        re = __ldg(uk4 + o);
        pe = pe_at(xa, ya, za);
      }
      T u, v, w, e, p, hh;
      cons_to_prim(r, ru, rv, rw, re, pe, u, v, w, e, p, hh);
      R(slot, 0, px, py) = r;
      R(slot, 1, px, py) = u;
      R(slot, 2, px, py) = v;
      R(slot, 3, px, py) = w;
      R(slot, 4, px, py) = e;
      R(slot, 5, px, py) = p;
      R(slot, 6, px, py) = hh;
    }
  };
  const int zfirst = z0 - ZLO - 1;
  auto slot_of = [&](int z) { return (z - zfirst) % RING; };

  // z-face above cell (tx, ty) of plane zc, i.e. face index zc + 1.
  auto zface = [&](int zc, T* f) {
    Prim<T> ql, qr;
#pragma unroll
    for (int v = 0; v < 7; ++v) {
      T s[NW];
#pragma unroll
      for (int k = 0; k < NW; ++k)
        s[k] = R(slot_of(zc + 1 - LO + k), v, HR + tx, HR + ty);
      T ng, ps;
      reconstruct<SCHEME>(s, a.limiter, ng, ps);
      set_var(ql, v, ng);
      set_var(qr, v, ps);
    }
    T pe = pe_at(x0 + tx + h, y0 + ty + h, zc + 1 + h);
    riemann<RIEMANN, T, 2>(ql, qr, pe, f);
    if constexpr (VISC) {
      const int sa = slot_of(zc), sb = slot_of(zc + 1);
      const int px = HR + tx, py = HR + ty;
      T ua[3], ub[3], ga[3][3], gb[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ua[c] = R(sa, 1 + c, px, py);
        ub[c] = R(sb, 1 + c, px, py);
      }
      // tangential x (rows) and y (cols); components c == t and c == 2.
      const T i2dx = T(2) * dx, i2dy = T(2) * dy;
      ga[0][0] = (R(sa, 1, px + 1, py) - R(sa, 1, px - 1, py)) / i2dx;
      gb[0][0] = (R(sb, 1, px + 1, py) - R(sb, 1, px - 1, py)) / i2dx;
      ga[0][2] = (R(sa, 3, px + 1, py) - R(sa, 3, px - 1, py)) / i2dx;
      gb[0][2] = (R(sb, 3, px + 1, py) - R(sb, 3, px - 1, py)) / i2dx;
      ga[1][1] = (R(sa, 2, px, py + 1) - R(sa, 2, px, py - 1)) / i2dy;
      gb[1][1] = (R(sb, 2, px, py + 1) - R(sb, 2, px, py - 1)) / i2dy;
      ga[1][2] = (R(sa, 3, px, py + 1) - R(sa, 3, px, py - 1)) / i2dy;
      gb[1][2] = (R(sb, 3, px, py + 1) - R(sb, 3, px, py - 1)) / i2dy;
      viscous_flux<T, 2>(R(sa, 0, px, py), R(sb, 0, px, py), ua, ub,
                         R(sa, 5, px, py), R(sb, 5, px, py), ga, gb, dz, nu,
                         inv_pr, f);
    }
  };

  // ---- warm-up: planes zfirst .. z0+ZHI-1 and the z-face below z0.
  for (int i = 0; i < RING; ++i) load_plane(zfirst + i, i);
  __syncthreads();
  const bool own = (x0 + tx < a.nx) && (y0 + ty < a.ny);
  T flo[5], fhi[5];
  if (own) zface(z0 - 1, flo);
  __syncthreads();

  double dtmin_local = 1e300;
  const double dt_d = a.dt ? *a.dt : 0.0;
  const T dt = T(dt_d);
  const T c0 = T(a.c0), c1 = T(a.c1);

  for (int zc = z0; zc < z1; ++zc) {
    // Plane zc+ZHI replaces plane zc-ZLO-1, last read before the previous
    // barrier.
    load_plane(zc + ZHI, slot_of(zc + ZHI));
    __syncthreads();
    const int cs = slot_of(zc);
    const int sm1 = slot_of(zc - 1), sp1 = slot_of(zc + 1);
    (void)sm1;
    (void)sp1;

    // ---- y-faces of plane zc: (TY+1) per row.
    for (int f = tid; f < TX * (TY + 1); f += NT) {
      const int fxx = f / (TY + 1), fyy = f - fxx * (TY + 1);
      if (x0 + fxx >= a.nx || y0 + fyy > a.ny) continue;
      Prim<T> ql, qr;
#pragma unroll
      for (int v = 0; v < 7; ++v) {
        T s[NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) s[k] = R(cs, v, HR + fxx, HR + fyy - LO + k);
        T ng, ps;
        reconstruct<SCHEME>(s, a.limiter, ng, ps);
        set_var(ql, v, ng);
        set_var(qr, v, ps);
      }
      T ff[5];
      T pe = pe_at(x0 + fxx + h, y0 + fyy + h, zc + h);
      riemann<RIEMANN, T, 1>(ql, qr, pe, ff);
      if constexpr (VISC) {
        const int px = HR + fxx, pa = HR + fyy - 1, pb = HR + fyy;
        T ua[3], ub[3], ga[3][3], gb[3][3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ua[c] = R(cs, 1 + c, px, pa);
          ub[c] = R(cs, 1 + c, px, pb);
        }
        const T i2dx = T(2) * dx, i2dz = T(2) * dz;
        ga[0][0] = (R(cs, 1, px + 1, pa) - R(cs, 1, px - 1, pa)) / i2dx;
        gb[0][0] = (R(cs, 1, px + 1, pb) - R(cs, 1, px - 1, pb)) / i2dx;
        ga[0][1] = (R(cs, 2, px + 1, pa) - R(cs, 2, px - 1, pa)) / i2dx;
        gb[0][1] = (R(cs, 2, px + 1, pb) - R(cs, 2, px - 1, pb)) / i2dx;
        ga[2][2] = (R(sp1, 3, px, pa) - R(sm1, 3, px, pa)) / i2dz;
        gb[2][2] = (R(sp1, 3, px, pb) - R(sm1, 3, px, pb)) / i2dz;
        ga[2][1] = (R(sp1, 2, px, pa) - R(sm1, 2, px, pa)) / i2dz;
        gb[2][1] = (R(sp1, 2, px, pb) - R(sm1, 2, px, pb)) / i2dz;
        viscous_flux<T, 1>(R(cs, 0, px, pa), R(cs, 0, px, pb), ua, ub,
                           R(cs, 5, px, pa), R(cs, 5, px, pb), ga, gb, dy, nu,
                           inv_pr, ff);
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) fy[(v * TX + fxx) * (TY + 1) + fyy] = ff[v];
    }

    // ---- x-faces of plane zc: (TX+1) rows of TY.
    for (int f = tid; f < (TX + 1) * TY; f += NT) {
      const int fxx = f / TY, fyy = f - fxx * TY;
      if (x0 + fxx > a.nx || y0 + fyy >= a.ny) continue;
      Prim<T> ql, qr;
#pragma unroll
      for (int v = 0; v < 7; ++v) {
        T s[NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) s[k] = R(cs, v, HR + fxx - LO + k, HR + fyy);
        T ng, ps;
        reconstruct<SCHEME>(s, a.limiter, ng, ps);
        set_var(ql, v, ng);
        set_var(qr, v, ps);
      }
      T ff[5];
      T pe = pe_at(x0 + fxx + h, y0 + fyy + h, zc + h);
      riemann<RIEMANN, T, 0>(ql, qr, pe, ff);
      if constexpr (VISC) {
        const int py = HR + fyy, pa = HR + fxx - 1, pb = HR + fxx;
        T ua[3], ub[3], ga[3][3], gb[3][3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ua[c] = R(cs, 1 + c, pa, py);
          ub[c] = R(cs, 1 + c, pb, py);
        }
        const T i2dy = T(2) * dy, i2dz = T(2) * dz;
        ga[1][1] = (R(cs, 2, pa, py + 1) - R(cs, 2, pa, py - 1)) / i2dy;
        gb[1][1] = (R(cs, 2, pb, py + 1) - R(cs, 2, pb, py - 1)) / i2dy;
        ga[1][0] = (R(cs, 1, pa, py + 1) - R(cs, 1, pa, py - 1)) / i2dy;
        gb[1][0] = (R(cs, 1, pb, py + 1) - R(cs, 1, pb, py - 1)) / i2dy;
        ga[2][2] = (R(sp1, 3, pa, py) - R(sm1, 3, pa, py)) / i2dz;
        gb[2][2] = (R(sp1, 3, pb, py) - R(sm1, 3, pb, py)) / i2dz;
        ga[2][0] = (R(sp1, 1, pa, py) - R(sm1, 1, pa, py)) / i2dz;
        gb[2][0] = (R(sp1, 1, pb, py) - R(sm1, 1, pb, py)) / i2dz;
        viscous_flux<T, 0>(R(cs, 0, pa, py), R(cs, 0, pb, py), ua, ub,
                           R(cs, 5, pa, py), R(cs, 5, pb, py), ga, gb, dx, nu,
                           inv_pr, ff);
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) fx[(v * (TX + 1) + fxx) * TY + fyy] = ff[v];
    }

    // ---- z-face above each owned column.
    if (own) zface(zc, fhi);
    __syncthreads();

    // ---- divergence, source and stage combination.
    if (own) {
      const int xa = x0 + tx + h, ya = y0 + ty + h, za = zc + h;
      const long long o = za * sz + xa * sx + ya;
      T src[5] = {T(0), T(0), T(0), T(0), T(0)};
      const T rho_c = R(cs, 0, HR + tx, HR + ty);
      if (a.gravity_mask) {
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (a.gravity_mask & (1 << d))
            src[1 + d] = rho_c * K<T>::grav() * T(a.g[d]);
      }
      T out[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        T rhs = src[v];
        rhs = rhs - (fx[(v * (TX + 1) + tx + 1) * TY + ty] -
                     fx[(v * (TX + 1) + tx) * TY + ty]) / dx;
        rhs = rhs - (fy[(v * TX + tx) * (TY + 1) + ty + 1] -
                     fy[(v * TX + tx) * (TY + 1) + ty]) / dy;
        rhs = rhs - (fhi[v] - flo[v]) / dz;
        const T* ukv = static_cast<const T*>(a.uk[v]);
        T r;
        if (a.mode == SWC_OUT_RHS) {
          r = rhs;
        } else if (a.mode == SWC_OUT_EULER) {
          r = __ldg(ukv + o) + rhs * dt;
        } else if (a.mode == SWC_OUT_CONVEX) {
          const T* u0v = static_cast<const T*>(a.u0[v]);
          r = __ldg(u0v + o) * c0 + (__ldg(ukv + o) + rhs * dt) * c1;
        } else {
          const T* u0v = static_cast<const T*>(a.u0[v]);
          r = c0 * (__ldg(u0v + o) + (__ldg(ukv + o) + dt * rhs));
        }
        out[v] = r;
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) static_cast<T*>(a.uout[v])[o] = out[v];
      if (a.dtmin_out) {
        T u, v, w, e, p, hh;
        cons_to_prim(out[0], out[1], out[2], out[3], out[4], pe_at(xa, ya, za),
                     u, v, w, e, p, hh);
        T c = sqrt_(K<T>::gamma() * p / out[0]);
        T l = min_(min_(dx / (abs_(u) + c), dy / (abs_(v) + c)),
                   dz / (abs_(w) + c));
        dtmin_local = fmin(dtmin_local, double(l));
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) flo[v] = fhi[v];
    }
  }

  if (a.dtmin_out) {
    // Block min of the CFL limits, then one atomic per CTA.
    __shared__ double red[32];
    double m = dtmin_local;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      m = fmin(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((tid & 31) == 0) red[tid >> 5] = m;
    __syncthreads();
    if (tid < 32) {
      m = (tid < NT / 32) ? red[tid] : 1e300;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1)
        m = fmin(m, __shfl_xor_sync(0xffffffffu, m, off));
      if (tid == 0 && m < 1e300) atomic_min_pos(a.dtmin_out, m);
    }
  }
}

}  // namespace swc
