// Halo fill of one dim for one grid (boundary.py:34-86, 464-539): the
// per-element routine shared by the single-grid and the batched passes.
#pragma once

#include "swc_physics.cuh"
#include "swirlc_b200.h"

namespace swc {

struct HaloField {
  void* f;
  int via_prim;
  SwcBC bc[2];
};
struct HaloArgs {
  int dim;  // 0 x, 1 y, 2 z
  int nf;
  HaloField fld[SWC_MAX_FIELDS];
  const void* rho;
  int nx, ny, nz, h;
  long long sx, sz;
};

// A batched pass: one member grid, up to 5 fields.
struct HaloMember {
  int dim;
  int nf;
  HaloField fld[5];
  const void* rho;
  int nx, ny, nz, h;
  long long sx, sz;
};

// Halo widths up to this take the path that reads every layer first.
constexpr int kHaloFast = 8;

// Halo cells of one (field, side, plane position) element t of the pass
// described by `a` (HaloArgs or HaloMember); t < plane * 2 * a.nf.
template <typename T, typename A>
__device__ __forceinline__ void halo_elem(const A& a, long long t) {
  // Axis sizes with halos, storage order (z, x, y).
  const int ext[3] = {a.nx + 2 * a.h, a.ny + 2 * a.h, a.nz + 2 * a.h};
  const long long stride[3] = {a.sx, 1, a.sz};
  const int d = a.dim;
  // Plane axes (A, B) in storage order of the two other axes.
  int ax_a, ax_b;
  if (d == 0) { ax_a = 2; ax_b = 1; }
  else if (d == 1) { ax_a = 2; ax_b = 0; }
  else { ax_a = 0; ax_b = 1; }
  const int na = ext[ax_a], nb = ext[ax_b];
  const long long plane = (long long)na * nb;
  const int n = ext[d] - 2 * a.h;
  {
    // Element t -> (field, side, plane position). 32-bit unsigned division
    // where the pass fits (a 64-bit division is a long software sequence).
    long long pb;
    int side, fi, ia, ib;
    if (plane * 2 * a.nf < (1LL << 32)) {
      const unsigned tt = (unsigned)t, pl = (unsigned)plane;
      const unsigned q = tt / pl;
      const unsigned p = tt - q * pl;
      side = (int)(q & 1u);
      fi = (int)(q >> 1);
      ia = (int)(p / (unsigned)nb);
      ib = (int)(p - (unsigned)ia * (unsigned)nb);
      pb = p;
    } else {
      pb = t % plane;
      side = (int)((t / plane) % 2);
      fi = (int)(t / (plane * 2));
      ia = (int)(pb / nb);
      ib = (int)(pb % nb);
    }
    const long long base = ia * stride[ax_a] + ib * stride[ax_b];
    const long long sd = stride[d];
    T* f = static_cast<T*>(a.fld[fi].f);
    const T* rho = static_cast<const T*>(a.rho);
    const bool prim = a.fld[fi].via_prim != 0;
    const SwcBC bc = a.fld[fi].bc[side];
    auto pv = [&](long long o) -> T {  // value the BC acts on
      if (!prim) return f[o];
      T r = rho[o];
      return r == T(0) ? T(0) : f[o] / r;
    };
    auto put = [&](long long o, T val) { f[o] = prim ? rho[o] * val : val; };
    auto dst = [&](int l) -> long long {
      return side == 0 ? base + (long long)l * sd
                       : base + (long long)(n + a.h + l) * sd;
    };
    if (a.h <= kHaloFast) {
      // Every layer's value is read before any is written: the compiler
      // cannot tell the written cells from the read ones, so reading and
      // writing layer by layer would cost one memory round trip per layer.
      T val[kHaloFast];
      bool set = true;
      if (bc.kind == SWC_BC_PERIODIC) {
#pragma unroll
        for (int l = 0; l < kHaloFast; ++l)
          if (l < a.h)
            val[l] = pv(side == 0 ? base + (long long)(l + n) * sd
                                  : base + (long long)(a.h + l) * sd);
      } else if (bc.kind == SWC_BC_DIRICHLET) {
        const T* pl = static_cast<const T*>(bc.planes);
#pragma unroll
        for (int l = 0; l < kHaloFast; ++l)
          if (l < a.h) val[l] = bc.per_layer ? pl[l * plane + pb] : T(bc.value);
      } else if (bc.kind == SWC_BC_NEUMANN) {
        // Layer l lies l+1 cells from the edge cell: value -+ (l+1)*inc,
        // accumulated one layer at a time.
        const T inc = T(bc.value);
        T v = pv(side == 0 ? base + (long long)a.h * sd
                           : base + (long long)(n + a.h - 1) * sd);
#pragma unroll
        for (int l = 0; l < kHaloFast; ++l) {
          v = side == 0 ? v - inc : v + inc;
          val[l] = v;
        }
      } else {
        set = false;
      }
      if (!set) return;
      // Neumann layer l is cell h-1-l on the low side, n+h+l on the high.
      auto cell = [&](int l) -> long long {
        return (bc.kind == SWC_BC_NEUMANN && side == 0)
                   ? base + (long long)(a.h - 1 - l) * sd
                   : dst(l);
      };
      if (prim) {
        T r[kHaloFast];
#pragma unroll
        for (int l = 0; l < kHaloFast; ++l)
          if (l < a.h) r[l] = rho[cell(l)];
#pragma unroll
        for (int l = 0; l < kHaloFast; ++l)
          if (l < a.h) f[cell(l)] = r[l] * val[l];
      } else {
#pragma unroll
        for (int l = 0; l < kHaloFast; ++l)
          if (l < a.h) f[cell(l)] = val[l];
      }
      return;
    }
    if (bc.kind == SWC_BC_PERIODIC) {
      for (int l = 0; l < a.h; ++l) {
        if (side == 0) put(base + l * sd, pv(base + (long long)(l + n) * sd));
        else put(base + (long long)(n + a.h + l) * sd, pv(base + (long long)(a.h + l) * sd));
      }
    } else if (bc.kind == SWC_BC_DIRICHLET) {
      const T* pl = static_cast<const T*>(bc.planes);
      for (int l = 0; l < a.h; ++l) {
        T val = bc.per_layer ? pl[l * plane + pb] : T(bc.value);
        put(dst(l), val);
      }
    } else if (bc.kind == SWC_BC_NEUMANN) {
      const T inc = T(bc.value);
      if (side == 0) {
        T v = pv(base + (long long)a.h * sd);
        for (int l = 0; l < a.h; ++l) {
          v = v - inc;
          put(base + (long long)(a.h - 1 - l) * sd, v);
        }
      } else {
        T v = pv(base + (long long)(n + a.h - 1) * sd);
        for (int l = 0; l < a.h; ++l) {
          v = v + inc;
          put(base + (long long)(n + a.h + l) * sd, v);
        }
      }
    }
  }
}

// Halo fill, in one pass, of fields whose every dim is periodic (clamp[d] =
// 0) or zero-gradient (Neumann with value 0 on both sides, clamp[d] = 1):
// each halo cell copies the interior cell it wraps to, or the edge cell it
// clamps to. The x, y, z passes of halo_kernel compose to exactly this copy
// when no halo is wider than the interior (each pass copies interior
// layers, a Neumann layer with increment 0 is its edge value, and a
// corner's value reaches it through the other dims' copies). Thread
// t < 2h planes of nxa*nya cells takes a whole z-halo plane cell; the rest
// take the x/y frame (2h full rows, then 2h cells of each interior row) of
// the interior planes. 32-bit indices (the caller checks the count).
//
// Element t of the halo shell (t < halo_shell_count) of the grid in `a`
// (HaloArgs or HaloMember).
// Padded coordinates (xa, ya, za) of element t of the halo shell.
__device__ __forceinline__ void shell_cell(int h, int nx, int ny, int nz,
                                           int t, int& xa, int& ya, int& za) {
  const int nxa = nx + 2 * h, nya = ny + 2 * h;
  const int plane = nxa * nya;
  const int frame = 2 * h * nya + nx * 2 * h;
  if (t < 2 * h * plane) {
    const int zi = t / plane, r = t - zi * plane;
    za = zi < h ? zi : nz + zi;
    xa = r / nya;
    ya = r - xa * nya;
  } else {
    const int u = t - 2 * h * plane;
    const int zi = u / frame;
    int r = u - zi * frame;
    za = h + zi;
    if (r < 2 * h * nya) {
      const int row = r / nya;
      ya = r - row * nya;
      xa = row < h ? row : nx + row;
    } else {
      r -= 2 * h * nya;
      const int q = r / (2 * h), j = r - q * (2 * h);
      xa = h + q;
      ya = j < h ? j : ny + j;
    }
  }
}

template <typename T, typename A>
__device__ __forceinline__ void halo_shell_elem(const A& a, int t, int clamp_x,
                                                int clamp_y, int clamp_z) {
  constexpr int NFMAX = sizeof(A::fld) / sizeof(A::fld[0]);
  const int h = a.h, nx = a.nx, ny = a.ny, nz = a.nz;
  int xa, ya, za;
  shell_cell(h, nx, ny, nz, t, xa, ya, za);
  auto src = [h](int c, int n, int clamp) {
    if (clamp) return c < h ? h : (c >= n + h ? n + h - 1 : c);
    return c < h ? c + n : (c >= n + h ? c - n : c);
  };
  const long long o = za * a.sz + xa * a.sx + ya;
  const long long os = src(za, nz, clamp_z) * a.sz +
                       src(xa, nx, clamp_x) * a.sx + src(ya, ny, clamp_y);
  // Every load before any store (the compiler cannot tell the fields apart).
  T v[NFMAX];
#pragma unroll
  for (int f = 0; f < NFMAX; ++f)
    if (f < a.nf) v[f] = static_cast<const T*>(a.fld[f].f)[os];
#pragma unroll
  for (int f = 0; f < NFMAX; ++f)
    if (f < a.nf) static_cast<T*>(a.fld[f].f)[o] = v[f];
}

// One-pass fill of fields whose every side is periodic, Dirichlet (a value
// or per-layer planes) or Neumann (an increment per layer), none of them
// given on a primitive variable, with no periodic dim narrower than the
// halo. The x, y, z passes of halo_kernel compose to this: a halo cell's
// value is made by the last pass whose dim has the cell in its halo.
// Walking the passes backwards from that one, a periodic dim moves the cell
// to the cell it wraps to, a Neumann dim moves it to its edge cell (that
// layer's increments are applied later), and a Dirichlet dim ends the walk
// with its layer's value at the cell's position; otherwise the walk ends at
// an interior cell. The value is then rebuilt forwards with the Neumann
// increments in pass order, one layer at a time as the passes add them, so
// the result is bit for bit that of the three passes.
struct ShellField {
  void* f;
  SwcBC bc[3][2];  // [x, y, z][low, high]; a periodic dim is so on both sides
};
struct ShellArgs {
  int nf;
  ShellField fld[SWC_MAX_FIELDS];
  int nx, ny, nz, h;
  long long sx, sz;
};

template <typename T>
__device__ __forceinline__ void halo_shell_bc_elem(const ShellArgs& a, int t) {
  const int h = a.h;
  const int n[3] = {a.nx, a.ny, a.nz};
  const int ext[3] = {a.nx + 2 * h, a.ny + 2 * h, a.nz + 2 * h};
  int c0[3];
  shell_cell(h, a.nx, a.ny, a.nz, t, c0[0], c0[1], c0[2]);
  // Every load before any store (the compiler cannot tell the fields
  // apart); the loads are of interior cells and planes, which no thread
  // writes.
  T v[SWC_MAX_FIELDS];
#pragma unroll
  for (int fi = 0; fi < SWC_MAX_FIELDS; ++fi) {
    if (fi >= a.nf) break;
    const ShellField& F = a.fld[fi];
    int c[3] = {c0[0], c0[1], c0[2]};
    // Neumann steps met on the way back: layers and side per dim.
    int nl[3] = {0, 0, 0}, ns[3] = {0, 0, 0};
    bool dir = false;
    T val = T(0);
#pragma unroll
    for (int d = 2; d >= 0; --d) {
      const int side = c[d] < h ? 0 : (c[d] >= n[d] + h ? 1 : -1);
      if (side < 0) continue;
      const SwcBC& b = side == 0 ? F.bc[d][0] : F.bc[d][1];
      if (b.kind == SWC_BC_PERIODIC) {
        c[d] = side == 0 ? c[d] + n[d] : c[d] - n[d];
      } else if (b.kind == SWC_BC_NEUMANN) {
        // Layer l lies l + 1 cells from the edge cell.
        ns[d] = side;
        nl[d] = side == 0 ? h - c[d] : c[d] - (n[d] + h) + 1;
        c[d] = side == 0 ? h : n[d] + h - 1;
      } else {
        // Dirichlet: layer 0 is the outermost on the low side, the
        // innermost on the high side; planes are [halo][A][B] with (A, B)
        // the other two dims in storage order (z, x, y).
        const int l = side == 0 ? c[d] : c[d] - n[d] - h;
        if (b.per_layer) {
          int ia, ib, na, nb;
          if (d == 0) { ia = c[2]; ib = c[1]; na = ext[2]; nb = ext[1]; }
          else if (d == 1) { ia = c[2]; ib = c[0]; na = ext[2]; nb = ext[0]; }
          else { ia = c[0]; ib = c[1]; na = ext[0]; nb = ext[1]; }
          val = static_cast<const T*>(b.planes)[(long long)l * na * nb +
                                                (long long)ia * nb + ib];
        } else {
          val = T(b.value);
        }
        dir = true;
        break;
      }
    }
    if (!dir)
      val = static_cast<const T*>(F.f)[c[2] * a.sz + c[0] * a.sx + c[1]];
    // Forwards: the Neumann steps in pass order x, y, z (only dims after a
    // Dirichlet one were walked, so only those have steps).
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T inc = T(ns[d] == 0 ? F.bc[d][0].value : F.bc[d][1].value);
      for (int l = 0; l < nl[d]; ++l) val = ns[d] == 0 ? val - inc : val + inc;
    }
    v[fi] = val;
  }
  const long long o = c0[2] * a.sz + c0[0] * a.sx + c0[1];
#pragma unroll
  for (int fi = 0; fi < SWC_MAX_FIELDS; ++fi)
    if (fi < a.nf) static_cast<T*>(a.fld[fi].f)[o] = v[fi];
}

// Cells of the halo shell of an (nx, ny, nz) grid with halo h.
inline long long halo_shell_count(int nx, int ny, int nz, int h) {
  const long long nxa = nx + 2LL * h, nya = ny + 2LL * h;
  return 2LL * h * nxa * nya + (long long)nz * (2LL * h * nya + 2LL * h * nx);
}

}  // namespace swc
