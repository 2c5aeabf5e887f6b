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
// memory; each step computes every y- and x-face of the centre plane into
// shared memory and the z-face above each column in registers (the face
// below is carried from the previous step), converts the next plane into a
// ring slot those faces do not read, and after the step's one barrier forms
// the divergence and the stage update of the centre plane. Each face flux is
// computed exactly once per CTA. x and y faces reconstruct both face states
// from the face's stencil; z faces take them from cell-centred
// reconstructions of the column's cells, one per cell, whose upper-face
// value is carried up the column. The primitives are reconstructed two at a
// time (f32x2 lanes), all with explicitly rounded operations.
#pragma once

#include <type_traits>

#include "swc_physics.cuh"
#include "swirlc_b200.h"

// Members per batched launch (the member table is a launch parameter).
#define SWC_BATCH_CHUNK 64

namespace swc {

struct StageArgs {
  int nx, ny, nz, halo;
  long long sx, sz;
  double dx, dy, dz;
  const void* uk[SWC_MAX_FIELDS];
  const void* u0[SWC_MAX_FIELDS];
  void* uout[SWC_MAX_FIELDS];
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

template <int SCHEME, bool VISC>
struct Geom {
  static constexpr int LO = Stencil<SCHEME>::LO;
  static constexpr int RI = Stencil<SCHEME>::RI;
  static constexpr int NW = LO + RI;
  // Cell-centred stencil v[c-CL .. c+CR] (z faces).
  static constexpr int CL = CellStencil<SCHEME>::CL;
  static constexpr int CR = CellStencil<SCHEME>::CR;
  static constexpr int CW = CL + CR + 1;
  static constexpr int cmax(int a, int b) { return a > b ? a : b; }
  static constexpr int NOFF = cmax(NW, CW);
  static constexpr int HR = cmax(cmax(LO, RI - 1), VISC ? 1 : 0);
  // Planes below / above the centre plane zc held in the ring: the cell
  // above (zc+1) is reconstructed along z while zc is processed, and the
  // first pass of a segment also reconstructs its own plane.
  static constexpr int ZLO = cmax(cmax(cmax(LO - 1, CL), VISC ? 1 : 0), 0);
  static constexpr int ZHI = cmax(cmax(cmax(RI, CR + 1), VISC ? 1 : 0), 1);
  // The next plane is converted while the faces of plane zc are still being
  // read, into the slot of plane zc-ZLO-SPARE. The faces read plane zc, the
  // planes from zc+1-CL up (the z reconstruction of cell zc+1) and, viscous,
  // zc-1 (tangential differences), so that slot is free when ZLO >= 1,
  // ZLO >= CL and, viscous, ZLO >= 2; otherwise one spare slot is added
  // (not loaded by the warm-up, so the halo depth the arrays need does not
  // change).
  static constexpr int SPARE =
      (ZLO >= 1 && ZLO >= CL && (!VISC || ZLO >= 2)) ? 0 : 1;
  static constexpr int RING = ZLO + 1 + ZHI + SPARE;
  // Halo layers the stored arrays need.
  static constexpr int NEED = cmax(HR, cmax(ZLO + 1, ZHI));
};

// Shared-memory layout. NS transported scalars and (HELP) the p_dyn helper
// add reconstructed variables to the 7 primitives rho, u, v, w, e, p, h.
template <typename T, int SCHEME, bool VISC, int TY, int TX, int NS = 0,
          bool HELP = false>
struct Layout {
  using G = Geom<SCHEME, VISC>;
  static constexpr int NV = 7 + NS + (HELP ? 1 : 0);   // ring variables
  static constexpr int NCS = 5 + NS + (HELP ? 1 : 0);  // staged fields
  static constexpr int NF = 5 + NS;                     // flux components
  static constexpr int PW = TY + 2 * G::HR;
  static constexpr int PH = TX + 2 * G::HR;
  static constexpr int PS = PW * PH;
  static constexpr int NT = TX * TY;
  static constexpr int PER = (PS + NT - 1) / NT;  // plane cells per thread
  static constexpr int RING_ELEMS = G::RING * NV * PS;
  static constexpr int STAGE_ELEMS = NCS * PS;
  // x- and y-face fluxes, two buffers each (planes alternate), so that
  // threads may start the next plane's faces while others still form the
  // update of this one. The z-face flux stays in the registers of the
  // thread that computes and uses it.
  static constexpr int FY_ELEMS = NF * TX * (TY + 1);
  static constexpr int FX_ELEMS = NF * (TX + 1) * TY;
  static constexpr size_t SMEM =
      sizeof(T) * (size_t)(RING_ELEMS + STAGE_ELEMS + 2 * (FY_ELEMS + FX_ELEMS));
};

// 4- or 8-byte asynchronous global->shared copy (LDGSTS), cached in L1 so
// the centre-plane reload of the stage update hits on chip.
template <typename T>
__device__ __forceinline__ void cp_async(T* smem, const T* gmem) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  if constexpr (sizeof(T) == 4) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s),
                 "l"(gmem));
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s),
                 "l"(gmem));
  }
}
// Hint that the line holding *p will be read soon (no register is used;
// callers pass only addresses they will load).
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];\n" ::"l"(p));
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// One CTA's work: the TY x TX column at (y0, x0), z segment zb of `a`.
// NS scalars, HELP (p_ref/rho_ref) and EXT (face and flux overrides from
// `ext` on the grid's boundary faces) are compiled in only where asked for.
template <typename T, int SCHEME, int RIEMANN, bool VISC, int TY, int TX,
          int NS = 0, bool HELP = false, bool EXT = false>
__device__ __forceinline__ void stage_body(const StageArgs& a,
                                           const SwcStageExt* ext, const int y0,
                                           const int x0, const int zb) {
  using G = Geom<SCHEME, VISC>;
  using L = Layout<T, SCHEME, VISC, TY, TX, NS, HELP>;
  constexpr int NV = L::NV, NCS = L::NCS, NF = L::NF;
  constexpr int LO = G::LO, NW = G::NW, HR = G::HR, ZLO = G::ZLO,
                ZHI = G::ZHI, RING = G::RING, SPARE = G::SPARE, CL = G::CL,
                CW = G::CW, NOFF = G::NOFF;
  constexpr int PW = L::PW, PH = L::PH, PS = L::PS, NT = L::NT, PER = L::PER;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = reinterpret_cast<T*>(smem_raw);
  T* stg = ring + L::RING_ELEMS;    // [NCS][PS] conserved plane in flight
  T* fy0 = stg + L::STAGE_ELEMS;    // [2][NF][TX][TY+1]
  T* fx0 = fy0 + 2 * L::FY_ELEMS;   // [2][NF][TX+1][TY]

  const int tid = threadIdx.x;
  // Cell of this thread. For TY = 16 a warp covers rows w and w + TX/2, whose
  // shared-memory rows are (TX/2)*PW floats apart: with PW = 22 and TX = 16
  // that is 176 = 16 (mod 32), so the two half-warps hit disjoint banks.
  int ty, tx;
  if constexpr (TY == 16 && TX % 2 == 0) {
    const int w = tid >> 5, lane = tid & 31;
    ty = lane & 15;
    tx = w + (lane >> 4) * (TX / 2);
  } else {
    ty = tid % TY;
    tx = tid / TY;
  }
  const int z0 = zb * a.zseg;
  const int z1 = min(z0 + a.zseg, a.nz);
  const int h = a.halo;
  const int nxa = a.nx + 2 * h, nya = a.ny + 2 * h;
  const long long sx = a.sx, sz = a.sz;

  const T* __restrict__ ukp[NCS];
#pragma unroll
  for (int v = 0; v < 5 + NS; ++v) ukp[v] = static_cast<const T*>(a.uk[v]);
  if constexpr (HELP) ukp[5 + NS] = static_cast<const T*>(ext->p_ref);
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
    return ring[((slot * NV + v) * PH + px) * PW + py];
  };
  // Plane cells this thread stages and converts: idx = tid + k*NT.
  auto cell_valid = [&](int idx, int& xa, int& ya) -> bool {
    const int px = idx / PW, py = idx - px * PW;
    xa = x0 - HR + px + h;
    ya = y0 - HR + py + h;
    return idx < PS && xa < nxa && ya < nya;
  };
  auto issue_plane = [&](int z) {
    const long long zo = (long long)(z + h) * sz;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int idx = tid + k * NT;
      int xa, ya;
      if (cell_valid(idx, xa, ya)) {
        const long long o = zo + xa * sx + ya;
#pragma unroll
        for (int v = 0; v < NCS; ++v) cp_async(stg + v * PS + idx, ukp[v] + o);
      }
    }
    cp_async_commit();
  };
  // Converts this thread's staged cells into ring slot `slot` (plane z).
  auto convert_plane = [&](int z, int slot) {
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int idx = tid + k * NT;
      if (idx >= PS) break;
      int xa, ya;
      T c[5] = {T(1), T(0), T(0), T(0), T(1)};
      T pe = T(0);
      if (cell_valid(idx, xa, ya)) {
#pragma unroll
        for (int v = 0; v < 5; ++v) c[v] = stg[v * PS + idx];
        pe = pe_at(xa, ya, z + h);
      }
      T u, vv, w, e, p, hh;
      cons_to_prim(c[0], c[1], c[2], c[3], c[4], pe, u, vv, w, e, p, hh);
      const int px = idx / PW, py = idx - px * PW;
      R(slot, 0, px, py) = c[0];
      R(slot, 1, px, py) = u;
      R(slot, 2, px, py) = vv;
      R(slot, 3, px, py) = w;
      R(slot, 4, px, py) = e;
      R(slot, 5, px, py) = p;
      R(slot, 6, px, py) = hh;
      if constexpr (NS > 0 || HELP) {
        const bool ok = cell_valid(idx, xa, ya);
        const T inv = T(1) / c[0];
#pragma unroll
        for (int k = 0; k < NS; ++k)
          R(slot, 7 + k, px, py) = ok ? inv * stg[(5 + k) * PS + idx] : T(0);
        if constexpr (HELP) {
          // p_dyn = p - p_ref, zero in the halo layers beyond the grid's
          // boundary (exchange_halos with DIRICHLET 0 on all sides).
          const int za = z + h;
          const bool out =
              (xa < h && ext->boundary[0][0]) ||
              (xa >= a.nx + h && ext->boundary[0][1]) ||
              (ya < h && ext->boundary[1][0]) ||
              (ya >= a.ny + h && ext->boundary[1][1]) ||
              (za < h && ext->boundary[2][0]) ||
              (za >= a.nz + h && ext->boundary[2][1]);
          R(slot, 7 + NS, px, py) =
              (ok && !out) ? p - stg[(5 + NS) * PS + idx] : T(0);
        }
      }
    }
  };
  const int zfirst = z0 - ZLO - 1;
  auto slot_of = [&](int z) { return (z - zfirst) % RING; };

  // ---- one face flux in the frame rotated so that the face normal is
  // axis 0: (n, t1, t2) = x:(x,y,z), y:(y,x,z), z:(z,x,y). The same code
  // serves all three face directions; only ring offsets differ.
  //   off[k]   ring offset of stencil cell k (cells i-LO .. i+RI-1) of var 0
  //   ta/tb    ring offsets of the t1-/t1+/t2-/t2+ neighbours of the cells
  //            a = i-1 and b = i (viscous cross derivatives)
  auto hsel = [&](int d) -> T { return d == 0 ? dx : (d == 1 ? dy : dz); };
  // Reciprocals of the launch-constant divisors h_d and 2 h_d.
  const T rdx = rcp_(dx), rdy = rcp_(dy), rdz = rcp_(dz);
  const T r2dx = rcp_(T(2) * dx), r2dy = rcp_(T(2) * dy), r2dz = rcp_(T(2) * dz);
  auto rsel = [&](int d) -> T { return d == 0 ? rdx : (d == 1 ? rdy : rdz); };
  auto r2sel = [&](int d) -> T { return d == 0 ? r2dx : (d == 1 ? r2dy : r2dz); };
  //   bside    EXT only: -1, or the side (0 low, 1 high) of the grid boundary
  //            this face lies on; pidx its index in a face plane [A][B]
  constexpr int NSA = NS > 0 ? NS : 1;
  // Every ring variable reconstructed at the ring offsets off[k]: with
  // CELL false the face form (stencil v[i-LO..i+RI-1] of face i-1/2; lo =
  // neg, hi = pos), with CELL true the cell form (stencil v[c-CL..c+CR]; lo
  // = value on the cell's lower face, hi = on its upper face). vel[] maps
  // the rotated velocity slots to ring variables. The 7 primitives run as
  // the pairs (rho, e), (u_n, u_t1), (u_t2, p) and h alone; each pair is
  // one two-lane instruction stream.
  auto recon_all = [&](auto cell_tag, const int* off, const int* vel,
                       Prim<T>& lo, Prim<T>& hi, T* phlo, T* phhi, T& pdlo,
                       T& pdhi) {
    constexpr bool CELL = decltype(cell_tag)::value;
    constexpr int NK = CELL ? CW : NW;
    using O2 = Two<T>;
    using O1 = One<T>;
    using V2 = typename O2::V;
    const int va[3] = {0, vel[0], vel[2]};
    const int vb[3] = {4, vel[1], 5};
    V2 rl[3], rh[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const T* ba = ring + va[j] * PS;
      const T* bb = ring + vb[j] * PS;
      V2 sv[NK];
#pragma unroll
      for (int k = 0; k < NK; ++k) sv[k] = O2::mk(ba[off[k]], bb[off[k]]);
      if constexpr (CELL) recon_cell<SCHEME, O2>(sv, a.limiter, rl[j], rh[j]);
      else recon_face<SCHEME, O2>(sv, a.limiter, rl[j], rh[j]);
    }
    lo.r = rl[0].x; lo.e = rl[0].y; lo.u[0] = rl[1].x;
    lo.u[1] = rl[1].y; lo.u[2] = rl[2].x; lo.p = rl[2].y;
    hi.r = rh[0].x; hi.e = rh[0].y; hi.u[0] = rh[1].x;
    hi.u[1] = rh[1].y; hi.u[2] = rh[2].x; hi.p = rh[2].y;
    auto one = [&](int var, T& l, T& r) {
      const T* base = ring + var * PS;
      T sv[NK];
#pragma unroll
      for (int k = 0; k < NK; ++k) sv[k] = base[off[k]];
      if constexpr (CELL) recon_cell<SCHEME, O1>(sv, a.limiter, l, r);
      else recon_face<SCHEME, O1>(sv, a.limiter, l, r);
    };
    one(6, lo.h, hi.h);
#pragma unroll
    for (int q = 0; q < NS; ++q) one(7 + q, phlo[q], phhi[q]);
    if constexpr (HELP) {
      one(7 + NS, pdlo, pdhi);
    } else {
      pdlo = lo.p;
      pdhi = hi.p;
    }
  };
  // z faces: the lower state of the face above plane zc is the upper-face
  // value of cell zc, carried from the previous plane's reconstruction.
  Prim<T> zq;
  T zph[NSA], zpd;
  auto face = [&](int dn, const int* off, int oa, int ob, const int* ta,
                  const int* tb, T pe, int bside, long long pidx, T* f) {
    const int t1 = dn == 0 ? 1 : 0, t2 = dn == 2 ? 1 : 2;
    const int vel[3] = {1 + dn, 1 + t1, 1 + t2};
    Prim<T> ql, qr;
    T phl[NSA], phr[NSA];
    T pdl, pdr;
    if (dn == 2) {
      // off[] is the cell stencil of cell zc+1: its lower-face value is the
      // upper state of this face, its upper-face value carries on.
      Prim<T> up;
      T phu[NSA], pdu;
      recon_all(std::true_type{}, off, vel, qr, up, phr, phu, pdr, pdu);
      ql = zq;
      zq = up;
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        phl[q] = zph[q];
        zph[q] = phu[q];
      }
      pdl = zpd;
      zpd = pdu;
    } else {
      recon_all(std::false_type{}, off, vel, ql, qr, phl, phr, pdl, pdr);
    }
    auto plane_val = [&](const SwcOverride& o) -> T {
      return o.plane ? static_cast<const T*>(o.plane)[pidx] : T(o.value);
    };
    if constexpr (EXT) {
      // Face BCs on both face states (boundary.py:247-337): a primitive is
      // set directly, a conservative one divided by the face density.
      if (bside >= 0) {
        const int n = ext->nface[dn][bside];
        for (int i = 0; i < n; ++i) {
          const SwcOverride& o = ext->face[dn][bside][i];
          const T val = plane_val(o);
          const bool cons = o.mode == SWC_FACE_CONSERVATIVE;
          const T vl = cons ? dnn(val, ql.r) : val;
          const T vr = cons ? dnn(val, qr.r) : val;
          const int c = o.var - 1;
          const int rr = c == dn ? 0 : (c == t1 ? 1 : 2);
#pragma unroll
          for (int r = 0; r < 3; ++r)
            if (o.var >= 1 && o.var <= 3 && r == rr) {
              ql.u[r] = vl;
              qr.u[r] = vr;
            }
          if (o.var == 4) {
            ql.e = vl;
            qr.e = vr;
          }
#pragma unroll
          for (int q = 0; q < NS; ++q)
            if (o.var == 5 + q) {
              phl[q] = vl;
              phr[q] = vr;
            }
        }
      }
    }
    T g[5];
    if constexpr (HELP) {
      if constexpr (RIEMANN == 0) hll_flux<T, 0>(ql, qr, pdl, pdr, pe, g);
      else hllc_flux<T, 0>(ql, qr, pdl, pdr, pe, g);
    } else {
      riemann<RIEMANN, T, 0>(ql, qr, pe, g);
    }
    T gs[NSA];
    if constexpr (NS > 0)
      scalar_fluxes<RIEMANN, T, 0>(ql, qr, pdl, pdr, pe, NS, phl, phr, gs);
    // Back to (x, y, z) momentum order.
    auto rot = [&](const T* gg, T* out) {
      out[0] = gg[0];
      out[1] = dn == 0 ? gg[1] : gg[2];
      out[2] = dn == 1 ? gg[1] : (dn == 0 ? gg[2] : gg[3]);
      out[3] = dn == 2 ? gg[1] : gg[3];
      out[4] = gg[4];
    };
    // Flux BCs of one type (boundary.py:89-183) on fb (x, y, z order) and
    // the scalar fluxes fbs.
    auto flux_bc = [&](int type, T* fb, T* fbs) {
      if (bside < 0) return;
      const int n = ext->nflux[dn][bside];
      for (int i = 0; i < n; ++i) {
        const SwcOverride& o = ext->flux[dn][bside][i];
        if (o.mode != type) continue;
        const T val = plane_val(o);
#pragma unroll
        for (int v = 0; v < 5; ++v)
          if (o.var == v) fb[v] = val;
#pragma unroll
        for (int q = 0; q < NS; ++q)
          if (o.var == 5 + q) fbs[q] = val;
      }
    };
    if constexpr (EXT) {
      T fc[5];
      rot(g, fc);
      flux_bc(SWC_FLUX_CONVECTIVE, fc, gs);
      T fv[5] = {T(0), T(0), T(0), T(0), T(0)};
      T fvs[NSA];
#pragma unroll
      for (int q = 0; q < NSA; ++q) fvs[q] = T(0);
      if constexpr (VISC) {
        T gv[5] = {T(0), T(0), T(0), T(0), T(0)};
        T ua[3], ub[3], ga[3][3], gb[3][3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          ua[c] = ring[vel[c] * PS + oa];
          ub[c] = ring[vel[c] * PS + ob];
        }
        const T i2t1 = T(2) * hsel(t1), i2t2 = T(2) * hsel(t2);
        const T ri2t1 = r2sel(t1), ri2t2 = r2sel(t2);
        ga[1][1] = divk(ring[vel[1] * PS + ta[1]] - ring[vel[1] * PS + ta[0]], i2t1, ri2t1);
        gb[1][1] = divk(ring[vel[1] * PS + tb[1]] - ring[vel[1] * PS + tb[0]], i2t1, ri2t1);
        ga[1][0] = divk(ring[vel[0] * PS + ta[1]] - ring[vel[0] * PS + ta[0]], i2t1, ri2t1);
        gb[1][0] = divk(ring[vel[0] * PS + tb[1]] - ring[vel[0] * PS + tb[0]], i2t1, ri2t1);
        ga[2][2] = divk(ring[vel[2] * PS + ta[3]] - ring[vel[2] * PS + ta[2]], i2t2, ri2t2);
        gb[2][2] = divk(ring[vel[2] * PS + tb[3]] - ring[vel[2] * PS + tb[2]], i2t2, ri2t2);
        ga[2][0] = divk(ring[vel[0] * PS + ta[3]] - ring[vel[0] * PS + ta[2]], i2t2, ri2t2);
        gb[2][0] = divk(ring[vel[0] * PS + tb[3]] - ring[vel[0] * PS + tb[2]], i2t2, ri2t2);
        viscous_flux<T, 0>(ring[oa], ring[ob], ua, ub, ring[5 * PS + oa],
                           ring[5 * PS + ob], ga, gb, hsel(dn), rsel(dn), nu,
                           inv_pr, gv);
        rot(gv, fv);
        flux_bc(SWC_FLUX_DIFFUSIVE, fv, fvs);
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) f[v] = fc[v] + fv[v];
#pragma unroll
      for (int q = 0; q < NS; ++q) f[5 + q] = gs[q] + fvs[q];
      flux_bc(SWC_FLUX_TOTAL, f, f + 5);
      return;
    }
    if constexpr (VISC) {
      T ua[3], ub[3], ga[3][3], gb[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ua[c] = ring[vel[c] * PS + oa];
        ub[c] = ring[vel[c] * PS + ob];
      }
      const T i2t1 = T(2) * hsel(t1), i2t2 = T(2) * hsel(t2);
      const T ri2t1 = r2sel(t1), ri2t2 = r2sel(t2);
      // Along t1: components t1 (rotated 1) and n (rotated 0).
      ga[1][1] = divk(ring[vel[1] * PS + ta[1]] - ring[vel[1] * PS + ta[0]], i2t1, ri2t1);
      gb[1][1] = divk(ring[vel[1] * PS + tb[1]] - ring[vel[1] * PS + tb[0]], i2t1, ri2t1);
      ga[1][0] = divk(ring[vel[0] * PS + ta[1]] - ring[vel[0] * PS + ta[0]], i2t1, ri2t1);
      gb[1][0] = divk(ring[vel[0] * PS + tb[1]] - ring[vel[0] * PS + tb[0]], i2t1, ri2t1);
      // Along t2: components t2 (rotated 2) and n.
      ga[2][2] = divk(ring[vel[2] * PS + ta[3]] - ring[vel[2] * PS + ta[2]], i2t2, ri2t2);
      gb[2][2] = divk(ring[vel[2] * PS + tb[3]] - ring[vel[2] * PS + tb[2]], i2t2, ri2t2);
      ga[2][0] = divk(ring[vel[0] * PS + ta[3]] - ring[vel[0] * PS + ta[2]], i2t2, ri2t2);
      gb[2][0] = divk(ring[vel[0] * PS + tb[3]] - ring[vel[0] * PS + tb[2]], i2t2, ri2t2);
      viscous_flux<T, 0>(ring[oa], ring[ob], ua, ub, ring[5 * PS + oa],
                         ring[5 * PS + ob], ga, gb, hsel(dn), rsel(dn), nu,
                         inv_pr, g);
    }
    rot(g, f);
#pragma unroll
    for (int q = 0; q < NS; ++q) f[5 + q] = gs[q];
  };

  const int SL = NV * PS;  // ring slot stride
  // Flux buffers of the plane in progress, and this thread's z-face flux.
  T* fx = fx0;
  T* fy = fy0;
  T fzr[NF];
  // Face of kind `kind` (0 = x-face at row fxx, 1 = y-face at column fyy,
  // 2 = z-face above plane zc) into the flux buffers (z: into fzr).
  auto do_face = [&](int kind, int zc, int fxx, int fyy) {
    int off[NOFF], ta[4], tb[4];
    T pe;
    T f[NF];
    // Grid-boundary side and face-plane index of this face (EXT only). The
    // face stored at i (interior numbering) is face i-1/2: i = 0 is the low
    // boundary, i = n the high one (boundary.py:140-183).
    int bside = -1;
    long long pidx = 0;
    if constexpr (EXT) {
      const int i = kind == 0 ? x0 + fxx : (kind == 1 ? y0 + fyy : zc + 1);
      const int n = kind == 0 ? a.nx : (kind == 1 ? a.ny : a.nz);
      if (i == 0 && ext->boundary[kind][0]) bside = 0;
      if (i == n && ext->boundary[kind][1]) bside = 1;
      if (kind == 0) pidx = (long long)(zc + h) * nya + (y0 + fyy + h);
      else if (kind == 1) pidx = (long long)(zc + h) * nxa + (x0 + fxx + h);
      else pidx = (long long)(x0 + fxx + h) * nya + (y0 + fyy + h);
    }
    if (kind == 2) {
      const int pos = (HR + fxx) * PW + HR + fyy;
#pragma unroll
      for (int k = 0; k < CW; ++k) off[k] = slot_of(zc + 1 - CL + k) * SL + pos;
      const int oa = slot_of(zc) * SL + pos, ob = slot_of(zc + 1) * SL + pos;
      ta[0] = oa - PW; ta[1] = oa + PW; ta[2] = oa - 1; ta[3] = oa + 1;
      tb[0] = ob - PW; tb[1] = ob + PW; tb[2] = ob - 1; tb[3] = ob + 1;
      pe = pe_at(x0 + fxx + h, y0 + fyy + h, zc + 1 + h);
      face(2, off, oa, ob, ta, tb, pe, bside, pidx, f);
#pragma unroll
      for (int v = 0; v < NF; ++v) fzr[v] = f[v];
    } else {
      const int cs = slot_of(zc) * SL;
      const int dm = (slot_of(zc - 1) - slot_of(zc)) * SL;
      const int dp = (slot_of(zc + 1) - slot_of(zc)) * SL;
      const int pos = cs + (HR + fxx) * PW + HR + fyy;
      const int st = kind == 0 ? PW : 1;     // normal stride
      const int s1 = kind == 0 ? 1 : PW;     // t1 stride (y for x-faces, x for y-faces)
#pragma unroll
      for (int k = 0; k < NW; ++k) off[k] = pos + (k - LO) * st;
      const int oa = pos - st, ob = pos;
      ta[0] = oa - s1; ta[1] = oa + s1; ta[2] = oa + dm; ta[3] = oa + dp;
      tb[0] = ob - s1; tb[1] = ob + s1; tb[2] = ob + dm; tb[3] = ob + dp;
      pe = pe_at(x0 + fxx + h, y0 + fyy + h, zc + h);
      face(kind, off, oa, ob, ta, tb, pe, bside, pidx, f);
      if (kind == 0) {
#pragma unroll
        for (int v = 0; v < NF; ++v) fx[(v * (TX + 1) + fxx) * TY + fyy] = f[v];
      } else {
#pragma unroll
        for (int v = 0; v < NF; ++v) fy[(v * TX + fxx) * (TY + 1) + fyy] = f[v];
      }
    }
  };

  // ---- warm-up: planes zfirst .. z0+ZHI-1 through the staging buffer (the
  // ring of the loop's first pass, zc = z0-1, which only computes the z-face
  // below the segment, so that every face of every segment comes from the
  // same code: results do not depend on where segments start); plane
  // z0+ZHI, converted during that pass, in flight.
  for (int i = 0; i < RING - SPARE; ++i) {
    issue_plane(zfirst + i);
    cp_async_wait_all();
    convert_plane(zfirst + i, i);
  }
  if (z0 < z1) issue_plane(z0 + ZHI);
  __syncthreads();
  const bool own = (x0 + tx < a.nx) && (y0 + ty < a.ny);
  T flo[NF];

  double dtmin_local = 1e300;
  const double dt_d = a.dt ? *a.dt : 0.0;
  const T dt = T(dt_d);
  const T c0 = T(a.c0), c1 = T(a.c1);
  const int xa_c = x0 + tx + h, ya_c = y0 + ty + h;

  // Per plane every owner computes three faces of its cell (z above, y and
  // x below); TY + TX threads also compute the tile's high x-row and high
  // y-column faces; owners of the last interior cell of a partial tile add
  // the face beyond it. The boundary block starts at a warp that moves on
  // from plane to plane (and from tile to tile), so its extra pass falls on
  // every SM sub-partition in turn instead of always on the last warp's.
  static_assert(TY + TX <= NT, "boundary faces need TY + TX threads");
  static_assert(NT % 32 == 0, "whole warps");
  constexpr int NWARP = NT / 32;
  const int tile_rot = x0 / TX + y0 / TY;
  const int nj = own ? 3 : 0;
  int bkind = -1, bx = 0, by = 0;
  auto boundary_faces = [&](int zc) {
    int wb = tid - ((zc - z0 + tile_rot) % NWARP) * 32;
    if (wb < 0) wb += NT;
    bkind = -1;
    if (wb < TY + TX) {
      if (wb < TY) { bkind = 0; bx = TX; by = wb; }
      else { bkind = 1; bx = wb - TY; by = TY; }
      if (bkind == 0 && !(x0 + TX <= a.nx && y0 + by < a.ny)) bkind = -1;
      if (bkind == 1 && !(y0 + TY <= a.ny && x0 + bx < a.nx)) bkind = -1;
    }
  };
  const bool ex_x = own && (x0 + tx + 1 == a.nx) && (tx + 1 < TX);
  const bool ex_y = own && (y0 + ty + 1 == a.ny) && (ty + 1 < TY);

  // One barrier per plane: faces of plane zc (x and y into flux buffer
  // zc & 1, z into registers), then the conversion of plane zc+ZHI+1 into
  // a slot no face of plane zc reads, the barrier, and the update of plane
  // zc, which reads no ring slot. A thread may start the faces of plane
  // zc+1 while others still update plane zc: they write the other flux
  // buffer, and buffer zc & 1 is next written after the following barrier.
  for (int zc = z0 - 1; zc < z1; ++zc) {
    const bool pre = zc < z0;  // only the z-face below the segment
    fx = fx0 + ((zc - z0 + 1) & 1) * L::FX_ELEMS;
    fy = fy0 + ((zc - z0 + 1) & 1) * L::FY_ELEMS;
    if (pre && own) {
      // Upper-face value of cell z0-1: the lower state of the segment's
      // first z face.
      const int pos = (HR + tx) * PW + HR + ty;
      int off[CW];
#pragma unroll
      for (int k = 0; k < CW; ++k) off[k] = slot_of(zc - CL + k) * SL + pos;
      const int vel[3] = {3, 1, 2};
      Prim<T> lf;
      T phlf[NSA], pdlf;
      recon_all(std::true_type{}, off, vel, lf, zq, phlf, zph, pdlf, zpd);
    }
    if (!pre) boundary_faces(zc);
    const int ntot = pre ? (own ? 1 : 0) : nj + (bkind >= 0) + ex_x + ex_y;
    for (int j = 0; j < ntot; ++j) {
      int kind, fxx, fyy;
      if (j < nj) {
        kind = 2 - j;  // z, y, x
        fxx = tx;
        fyy = ty;
      } else {
        int e = j - nj;
        if (bkind >= 0 && e == 0) {
          kind = bkind; fxx = bx; fyy = by;
        } else {
          if (bkind >= 0) --e;
          if (e == 0 && ex_x) { kind = 0; fxx = tx + 1; fyy = ty; }
          else { kind = 1; fxx = tx; fyy = ty + 1; }
        }
      }
      do_face(kind, zc, fxx, fyy);
    }
    // The cell's density for the gravity source, read while plane zc's
    // slot is certain to hold it (before the barrier).
    const T rho_cell =
        (a.gravity_mask && own && !pre) ? R(slot_of(zc), 0, HR + tx, HR + ty)
                                        : T(0);
    // Plane zc+ZHI+1 (staged during the previous plane) replaces the slot
    // of plane zc-ZLO-SPARE, which no face of plane zc reads. The first
    // pass also read plane zc-CL (its own cell's reconstruction), which can
    // be that plane: there the other threads' reads are waited for first.
    if (zc + 1 < z1) {
      if (pre) __syncthreads();
      cp_async_wait_all();
      convert_plane(zc + ZHI + 1, slot_of(zc + ZHI + 1));
      if (zc + 2 < z1) issue_plane(zc + ZHI + 2);
    }
    __syncthreads();
    if (pre) {
      if (own) {
#pragma unroll
        for (int v = 0; v < NF; ++v) flo[v] = fzr[v];
      }
      continue;
    }

    // ---- divergence, source and stage combination.
    if (own) {
      const int za = zc + h;
      const long long o = za * sz + (long long)xa_c * sx + ya_c;
      T ukc[NF], u0c[NF];
#pragma unroll
      for (int v = 0; v < NF; ++v) {
        ukc[v] = __ldg(ukp[v] + o);
        u0c[v] = (a.mode >= SWC_OUT_CONVEX)
                     ? __ldg(static_cast<const T*>(a.u0[v]) + o)
                     : T(0);
      }
      T src[5] = {T(0), T(0), T(0), T(0), T(0)};
      if (a.gravity_mask) {
        // Buoyancy acts on rho, or on rho - rho_ref with helper states.
        T rho_c = rho_cell;
        if constexpr (HELP)
          rho_c = rho_c - __ldg(static_cast<const T*>(ext->rho_ref) + o);
#pragma unroll
        for (int d = 0; d < 3; ++d)
          if (a.gravity_mask & (1 << d))
            src[1 + d] = rho_c * K<T>::grav() * T(a.g[d]);
      }
      T out[NF];
#pragma unroll
      for (int v = 0; v < NF; ++v) {
        const T fhi = fzr[v];
        T rhs = v < 5 ? src[v] : T(0);
        rhs = rhs - divk((fx[(v * (TX + 1) + tx + 1) * TY + ty] -
                     fx[(v * (TX + 1) + tx) * TY + ty]), dx, rdx);
        rhs = rhs - divk((fy[(v * TX + tx) * (TY + 1) + ty + 1] -
                     fy[(v * TX + tx) * (TY + 1) + ty]), dy, rdy);
        rhs = rhs - divk(fhi - flo[v], dz, rdz);
        flo[v] = fhi;
        T r;
        if (a.mode == SWC_OUT_RHS) {
          r = rhs;
        } else if (a.mode == SWC_OUT_EULER) {
          r = ukc[v] + rhs * dt;
        } else if (a.mode == SWC_OUT_CONVEX) {
          r = u0c[v] * c0 + (ukc[v] + rhs * dt) * c1;
        } else {
          r = c0 * (u0c[v] + (ukc[v] + dt * rhs));
        }
        out[v] = r;
      }
#pragma unroll
      for (int v = 0; v < NF; ++v) static_cast<T*>(a.uout[v])[o] = out[v];
      if (a.dtmin_out) {
        T u, v, w, e, p, hh;
        cons_to_prim(out[0], out[1], out[2], out[3], out[4],
                     pe_at(xa_c, ya_c, za), u, v, w, e, p, hh);
        T c = sqrt_(K<T>::gamma() * p / out[0]);
        T l = min_(min_(dx / (abs_(u) + c), dy / (abs_(v) + c)),
                   dz / (abs_(w) + c));
        dtmin_local = fmin(dtmin_local, cfl_limit_or_flag(out[0], p, out[4], l));
      }
    }
  }
  cp_async_wait_all();

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

// Resident CTAs per SM the register budget is set for: the inviscid MUSCL
// stage in single precision is light enough (shared memory 70 KB) for three.
template <typename T, int SCHEME, bool VISC>
constexpr int stage_min_blocks() {
  return sizeof(T) == 4 ? ((SCHEME == 2 && !VISC) ? 3 : 2) : 1;
}

template <typename T, int SCHEME, int RIEMANN, bool VISC, int TY, int TX>
__global__ void __launch_bounds__(TY* TX, (stage_min_blocks<T, SCHEME, VISC>()))
    stage_kernel(const StageArgs a) {
  stage_body<T, SCHEME, RIEMANN, VISC, TY, TX>(a, nullptr, blockIdx.x * TY,
                                               blockIdx.y * TX, blockIdx.z);
}

// Extended stage: NS transported scalars, HELP reference states, face and
// flux overrides on the grid boundary (one CTA per SM: the ring is larger).
template <typename T, int SCHEME, int RIEMANN, bool VISC, int TY, int TX,
          int NS, bool HELP>
__global__ void __launch_bounds__(TY* TX, 1)
    stage_kernel_ext(const StageArgs a, const SwcStageExt e) {
  stage_body<T, SCHEME, RIEMANN, VISC, TY, TX, NS, HELP, true>(
      a, &e, blockIdx.x * TY, blockIdx.y * TX, blockIdx.z);
}

// Batched stage: the CTAs of up to SWC_BATCH_CHUNK independent grids in one
// launch. CTA t belongs to the member m with pre[m] <= t < pre[m+1]; its
// tiles are numbered y fastest, then x, then z segment. The member table
// travels in the launch parameters, so the launch needs no device memory
// of its own and is captured whole by a CUDA graph.
struct StageBatch {
  int n;
  int pre[SWC_BATCH_CHUNK + 1];
  StageArgs m[SWC_BATCH_CHUNK];
};

template <typename T, int SCHEME, int RIEMANN, bool VISC, int TY, int TX>
__global__ void __launch_bounds__(TY* TX, sizeof(T) == 4 ? 2 : 1)
    stage_batch_kernel(const StageBatch b) {
  const int t = blockIdx.x;
  int lo = 0, hi = b.n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (b.pre[mid] <= t) lo = mid;
    else hi = mid;
  }
  // The member's record, copied to shared memory once per CTA, is read at
  // fixed addresses (no register holds a per-member offset).
  static_assert(sizeof(StageArgs) % 8 == 0, "StageArgs is copied as words");
  __shared__ StageArgs sa;
  {
    const long long* src = reinterpret_cast<const long long*>(&b.m[lo]);
    long long* dst = reinterpret_cast<long long*>(&sa);
    for (int i = threadIdx.x; i < (int)(sizeof(StageArgs) / 8); i += blockDim.x)
      dst[i] = src[i];
  }
  __syncthreads();
  const int local = t - b.pre[lo];
  const int nby = (sa.ny + TY - 1) / TY, nbx = (sa.nx + TX - 1) / TX;
  const int by = local % nby, rest = local / nby;
  stage_body<T, SCHEME, RIEMANN, VISC, TY, TX>(sa, nullptr, by * TY,
                                               (rest % nbx) * TX, rest / nbx);
}

}  // namespace swc
