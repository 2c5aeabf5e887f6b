// C-ABI entry points of libswirlc_b200 (declared in include/swirlc_b200.h)
// and the small kernels behind them: halo fill, CFL reduction, device clock,
// and the unit-level kernels (reconstruction, pointwise Riemann flux, wave
// speeds, stencils, stage algebra).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>

#include "swc_halo.cuh"
#include "swc_launch.h"
#include "swirlc_b200.h"

namespace swc {

static thread_local std::string g_last_error;
static thread_local int64_t g_launches = 0;

void note_launch(int n) { g_launches += n; }

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int record_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

static int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(SWC_ERR_LAUNCH, "%s: %s", what, cudaGetErrorString(e));
  return SWC_OK;
}

int check_grid(const SwcGrid* g) {
  if (!g) return fail(SWC_ERR_ARG, "grid is NULL");
  if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0 || g->halo < 0)
    return fail(SWC_ERR_ARG, "bad grid sizes nx=%d ny=%d nz=%d halo=%d", g->nx,
                g->ny, g->nz, g->halo);
  const int64_t nya = g->ny + 2 * g->halo, nxa = g->nx + 2 * g->halo;
  if (g->sx < nya || g->sz < g->sx * nxa)
    return fail(SWC_ERR_ARG, "bad strides sx=%lld sz=%lld", (long long)g->sx,
                (long long)g->sz);
  return SWC_OK;
}

static bool dtype_ok(int d) { return d == SWC_F32 || d == SWC_F64; }

// ---------------------------------------------------------------------------
// Halo fill (boundary.py:34-86, 464-539).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void halo_kernel(const HaloArgs a) {
  const int ext[3] = {a.nx + 2 * a.h, a.ny + 2 * a.h, a.nz + 2 * a.h};
  const int d = a.dim;
  const long long plane = (long long)ext[(d + 1) % 3] * ext[(d + 2) % 3];
  const long long total = plane * 2 * a.nf;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
       t < total; t += (long long)gridDim.x * blockDim.x)
    halo_elem<T>(a, t);
}

// One-pass halo fill of one grid (halo_shell_elem, swc_halo.cuh).
template <typename T>
__global__ void halo_periodic_kernel(const HaloArgs a, int total,
                                     int clamp_x, int clamp_y, int clamp_z) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < total) halo_shell_elem<T>(a, t, clamp_x, clamp_y, clamp_z);
}

// One-pass halo fill composing periodic, Dirichlet and Neumann sides
// (halo_shell_bc_elem, swc_halo.cuh).
template <typename T>
__global__ void halo_shell_kernel(const ShellArgs a, int total) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < total) halo_shell_bc_elem<T>(a, t);
}

// ---------------------------------------------------------------------------
// CFL reduction, device clock.
// ---------------------------------------------------------------------------
struct CflArgs {
  const void* u[5];
  const void* pe[3];
  int has_pe;
  int nx, ny, nz, h;
  long long sx, sz;
  double dx, dy, dz;
  double* out;
};

template <typename T>
__global__ void cfl_kernel(const CflArgs a) {
  const long long n = (long long)a.nx * a.ny * a.nz;
  double m = 1e300;
  const T* u0 = static_cast<const T*>(a.u[0]);
  const T* u1 = static_cast<const T*>(a.u[1]);
  const T* u2 = static_cast<const T*>(a.u[2]);
  const T* u3 = static_cast<const T*>(a.u[3]);
  const T* u4 = static_cast<const T*>(a.u[4]);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(t % a.ny);
    const int x = (int)((t / a.ny) % a.nx);
    const int z = (int)(t / ((long long)a.ny * a.nx));
    const int xa = x + a.h, ya = y + a.h, za = z + a.h;
    const long long o = za * a.sz + xa * a.sx + ya;
    T pe = T(0);
    if (a.has_pe) {
      const T* px = static_cast<const T*>(a.pe[0]);
      const T* py = static_cast<const T*>(a.pe[1]);
      const T* pz = static_cast<const T*>(a.pe[2]);
      pe = (-(px ? px[xa] : T(0)) - (py ? py[ya] : T(0))) - (pz ? pz[za] : T(0));
    }
    T uu, vv, ww, e, p, hh;
    T r = u0[o];
    cons_to_prim(r, u1[o], u2[o], u3[o], u4[o], pe, uu, vv, ww, e, p, hh);
    T c = sqrt_(K<T>::gamma() * p / r);
    T l = min_(min_(T(a.dx) / (abs_(uu) + c), T(a.dy) / (abs_(vv) + c)),
               T(a.dz) / (abs_(ww) + c));
    m = fmin(m, cfl_limit_or_flag(r, p, u4[o], l));
  }
  __shared__ double red[32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
    m = fmin(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = (threadIdx.x < blockDim.x / 32) ? red[threadIdx.x] : 1e300;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      m = fmin(m, __shfl_xor_sync(0xffffffffu, m, off));
    if (threadIdx.x == 0 && m < 1e300) atomic_min_pos(a.out, m);
  }
}

__global__ void clock_begin_kernel(SwcClock* c) { clock_begin(c); }

__global__ void clock_end_kernel(SwcClock* c) { clock_end(c); }

// ---------------------------------------------------------------------------
// Unit-level kernels.
// ---------------------------------------------------------------------------
struct Geo3 {
  int nxa, nya, nza;  // extents with halos
  long long sx, sz;
};

__device__ __forceinline__ void unflat(const Geo3& g, long long t, int& x,
                                       int& y, int& z) {
  y = (int)(t % g.nya);
  x = (int)((t / g.nya) % g.nxa);
  z = (int)(t / ((long long)g.nya * g.nxa));
}

template <typename T, int S>
__global__ void recon_kernel(Geo3 g, int dim, int limiter, const T* v, T* neg,
                             T* pos) {
  constexpr int LO = Stencil<S>::LO, RI = Stencil<S>::RI;
  const long long n = (long long)g.nxa * g.nya * g.nza;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    unflat(g, t, x, y, z);
    const int idx = dim == 0 ? x : (dim == 1 ? y : z);
    const int ext = dim == 0 ? g.nxa : (dim == 1 ? g.nya : g.nza);
    const long long st = dim == 0 ? g.sx : (dim == 1 ? 1 : g.sz);
    const long long o = z * g.sz + x * g.sx + y;
    if (idx - LO < 0 || idx + RI - 1 >= ext) {
      neg[o] = T(0);
      pos[o] = T(0);
      continue;
    }
    T s[LO + RI];
#pragma unroll
    for (int k = 0; k < LO + RI; ++k) s[k] = v[o + (k - LO) * st];
    T a, b;
    recon_face<S, One<T>>(s, limiter, a, b);
    neg[o] = a;
    pos[o] = b;
  }
}

struct PointArgs {
  long long n;
  int ns;  // transported scalars
  const void* ql[7 + 3];
  const void* qr[7 + 3];
  const void* pdl;
  const void* pdr;
  const void* pe;
  void* out[5 + 3];
  void* sl;
  void* sm;
  void* sr;
};

template <typename T, int D>
__device__ __forceinline__ void load_prim(const void* const* q, long long i,
                                          Prim<T>& p) {
  p.r = static_cast<const T*>(q[0])[i];
  p.u[0] = static_cast<const T*>(q[1])[i];
  p.u[1] = static_cast<const T*>(q[2])[i];
  p.u[2] = static_cast<const T*>(q[3])[i];
  p.e = static_cast<const T*>(q[4])[i];
  p.p = static_cast<const T*>(q[5])[i];
  p.h = static_cast<const T*>(q[6])[i];
}

// Pointwise flux; transported scalars phi follow the generic branches of
// the physical flux (m*phi, compressible_navier_stokes.py:419-427), of HLL
// (hll.py:159-170) and of the HLLC star flux (hllc.py:182-192).
template <typename T, int RM, int D>
__global__ void riemann_kernel(const PointArgs a) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n;
       i += (long long)gridDim.x * blockDim.x) {
    Prim<T> l, r;
    load_prim<T, D>(a.ql, i, l);
    load_prim<T, D>(a.qr, i, r);
    T pdl = a.pdl ? static_cast<const T*>(a.pdl)[i] : l.p;
    T pdr = a.pdr ? static_cast<const T*>(a.pdr)[i] : r.p;
    T pe = a.pe ? static_cast<const T*>(a.pe)[i] : T(0);
    T f[5];
    if constexpr (RM == 0) hll_flux<T, D>(l, r, pdl, pdr, pe, f);
    else hllc_flux<T, D>(l, r, pdl, pdr, pe, f);
#pragma unroll
    for (int k = 0; k < 5; ++k) static_cast<T*>(a.out[k])[i] = f[k];
    if (a.ns > 0) {
      T phl[3], phr[3], fs[3];
      for (int k = 0; k < a.ns; ++k) {
        phl[k] = static_cast<const T*>(a.ql[7 + k])[i];
        phr[k] = static_cast<const T*>(a.qr[7 + k])[i];
      }
      scalar_fluxes<RM, T, D>(l, r, pdl, pdr, pe, a.ns, phl, phr, fs);
      for (int k = 0; k < a.ns; ++k) static_cast<T*>(a.out[5 + k])[i] = fs[k];
    }
  }
}

template <typename T, int D>
__global__ void speeds_kernel(const PointArgs a) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < a.n;
       i += (long long)gridDim.x * blockDim.x) {
    Prim<T> l, r;
    load_prim<T, D>(a.ql, i, l);
    load_prim<T, D>(a.qr, i, r);
    T pe = a.pe ? static_cast<const T*>(a.pe)[i] : T(0);
    T s_l, s_r;
    hll_speeds<T, D>(l, r, pe, s_l, s_r);
    static_cast<T*>(a.sl)[i] = s_l;
    static_cast<T*>(a.sr)[i] = s_r;
    if (a.sm) static_cast<T*>(a.sm)[i] = hllc_contact<T, D>(l, r, s_l, s_r);
  }
}

template <typename T>
__global__ void stencil_kernel(Geo3 g, int op, int dim, double hd, const T* f,
                               T* out) {
  const long long n = (long long)g.nxa * g.nya * g.nza;
  const T h = T(hd);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    unflat(g, t, x, y, z);
    const int idx = dim == 0 ? x : (dim == 1 ? y : z);
    const int ext = dim == 0 ? g.nxa : (dim == 1 ? g.nya : g.nza);
    const long long st = dim == 0 ? g.sx : (dim == 1 ? 1 : g.sz);
    const long long o = z * g.sz + x * g.sx + y;
    const bool has_m = idx - 1 >= 0, has_p = idx + 1 < ext;
    T r = T(0);
    if (op == 0) { if (has_p) r = (f[o + st] - f[o]) / h; }
    else if (op == 1) { if (has_m) r = (f[o] - f[o - st]) / h; }
    else if (op == 2) { if (has_m && has_p) r = (f[o + st] - f[o - st]) / (T(2) * h); }
    else { if (has_m) r = T(0.5) * (f[o - st] + f[o]); }
    out[o] = r;
  }
}

template <typename T>
__global__ void combine_kernel(long long n, int mode, double c0d, double c1d,
                               const double* dtp, const T* u0, const T* uk,
                               const T* l, T* out) {
  const T dt = T(*dtp), c0 = T(c0d), c1 = T(c1d);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    T r;
    if (mode == SWC_OUT_EULER) r = uk[i] + l[i] * dt;
    else if (mode == SWC_OUT_CONVEX) r = u0[i] * c0 + (uk[i] + l[i] * dt) * c1;
    else r = c0 * (u0[i] + (uk[i] + dt * l[i]));
    out[i] = r;
  }
}

static unsigned blocks_for(long long n, int threads = 256) {
  long long b = (n + threads - 1) / threads;
  return (unsigned)std::max<long long>(1, std::min<long long>(b, 148 * 32));
}

// Viscous terms of every face i-1/2 of a whole array with the fused stage's
// face routine: viscous_flux in the frame rotated so that the face normal is
// axis 0, with the same launch-constant reciprocals, so a value here is bit
// for bit the viscous part the stage kernel forms on that face.
struct ViscArgs {
  Geo3 g;
  int what;
  const void* q[5];   // rho, u, v, w, p
  const void* rf[3];  // face densities (SWC_VISC_STRESS)
  double h[3];
  double nu, pr;
  void* out[15];
};

template <typename T>
__global__ void viscous_terms_kernel(const ViscArgs a) {
  const Geo3& g = a.g;
  const long long n = (long long)g.nxa * g.nya * g.nza;
  const T* qv[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) qv[v] = static_cast<const T*>(a.q[v]);
  const T h[3] = {T(a.h[0]), T(a.h[1]), T(a.h[2])};
  const T rh[3] = {rcp_(h[0]), rcp_(h[1]), rcp_(h[2])};
  const T r2h[3] = {rcp_(T(2) * h[0]), rcp_(T(2) * h[1]), rcp_(T(2) * h[2])};
  const T nu = a.what == SWC_VISC_STRAIN ? T(0.5) : T(a.nu);
  const T inv_pr = T(1.0 / a.pr);
  const bool zero_vel = a.what == SWC_VISC_HEAT;
  const bool cell_rho_p = a.what == SWC_VISC_FLUX || a.what == SWC_VISC_HEAT;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    unflat(g, t, x, y, z);
    const long long o = z * g.sz + x * g.sx + y;
    const int c3[3] = {x, y, z};
    const int ext[3] = {g.nxa, g.nya, g.nza};
    const long long st[3] = {g.sx, 1, g.sz};
#pragma unroll
    for (int dn = 0; dn < 3; ++dn) {
      const int t1 = dn == 0 ? 1 : 0, t2 = dn == 2 ? 1 : 2;
      // The heat flux reads only the two cells of the face; the other
      // quantities also read their tangential neighbours.
      const bool ok = c3[dn] >= 1 &&
                      (zero_vel || (c3[t1] >= 1 && c3[t1] + 1 < ext[t1] &&
                                    c3[t2] >= 1 && c3[t2] + 1 < ext[t2]));
      T fo[5] = {T(0), T(0), T(0), T(0), T(0)};
      if (ok) {
        const long long ob = o, oa = o - st[dn];
        const int vel[3] = {1 + dn, 1 + t1, 1 + t2};
        T ua[3], ub[3], ga[3][3] = {}, gb[3][3] = {};
        if (!zero_vel) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            ua[c] = qv[vel[c]][oa];
            ub[c] = qv[vel[c]][ob];
          }
          const T i2t1 = T(2) * h[t1], i2t2 = T(2) * h[t2];
          const long long s1 = st[t1], s2 = st[t2];
          ga[1][1] = divk(qv[vel[1]][oa + s1] - qv[vel[1]][oa - s1], i2t1, r2h[t1]);
          gb[1][1] = divk(qv[vel[1]][ob + s1] - qv[vel[1]][ob - s1], i2t1, r2h[t1]);
          ga[1][0] = divk(qv[vel[0]][oa + s1] - qv[vel[0]][oa - s1], i2t1, r2h[t1]);
          gb[1][0] = divk(qv[vel[0]][ob + s1] - qv[vel[0]][ob - s1], i2t1, r2h[t1]);
          ga[2][2] = divk(qv[vel[2]][oa + s2] - qv[vel[2]][oa - s2], i2t2, r2h[t2]);
          gb[2][2] = divk(qv[vel[2]][ob + s2] - qv[vel[2]][ob - s2], i2t2, r2h[t2]);
          ga[2][0] = divk(qv[vel[0]][oa + s2] - qv[vel[0]][oa - s2], i2t2, r2h[t2]);
          gb[2][0] = divk(qv[vel[0]][ob + s2] - qv[vel[0]][ob - s2], i2t2, r2h[t2]);
        } else {
#pragma unroll
          for (int c = 0; c < 3; ++c) ua[c] = ub[c] = T(0);
        }
        T ra, rb;
        if (a.what == SWC_VISC_STRAIN) {
          ra = rb = T(1);
        } else if (a.what == SWC_VISC_STRESS) {
          ra = rb = static_cast<const T*>(a.rf[dn])[ob];
        } else {
          ra = qv[0][oa];
          rb = qv[0][ob];
        }
        const T pa = cell_rho_p ? qv[4][oa] : T(1);
        const T pb = cell_rho_p ? qv[4][ob] : T(1);
        T f[5] = {T(0), T(0), T(0), T(0), T(0)};
        viscous_flux<T, 0>(ra, rb, ua, ub, pa, pb, ga, gb, h[dn], rh[dn], nu,
                           inv_pr, f);
        // Back to (x, y, z) momentum order.
        fo[1] = dn == 0 ? f[1] : f[2];
        fo[2] = dn == 1 ? f[1] : (dn == 0 ? f[2] : f[3]);
        fo[3] = dn == 2 ? f[1] : f[3];
        fo[4] = f[4];
      }
      if (a.what == SWC_VISC_FLUX) {
#pragma unroll
        for (int k = 0; k < 5; ++k) static_cast<T*>(a.out[dn * 5 + k])[o] = fo[k];
      } else if (a.what == SWC_VISC_HEAT) {
        static_cast<T*>(a.out[dn])[o] = fo[4];
      } else {
        // tau_{c, dn} (strain: S_{c, dn}) = -(momentum flux c across dn).
#pragma unroll
        for (int c = 0; c < 3; ++c) static_cast<T*>(a.out[c * 3 + dn])[o] = -fo[1 + c];
      }
    }
  }
}

}  // namespace swc

using namespace swc;

extern "C" {

int swc_abi_version(void) { return SWC_ABI_VERSION; }

int swc_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return (int)g_last_error.size();
  size_t n = std::min(len - 1, g_last_error.size());
  memcpy(buf, g_last_error.data(), n);
  buf[n] = 0;
  return (int)n;
}

int64_t swc_launch_count(void) { return g_launches; }

int swc_halo_fill(const SwcGrid* grid, int32_t dtype, int32_t nfields,
                  void* const* fields, const SwcFieldBC* bcs,
                  int32_t rho_index, void* stream) {
  swc::NvtxRange nvtx_range_("swc_halo_fill");
  int st = check_grid(grid);
  if (st) return st;
  if (!dtype_ok(dtype)) return fail(SWC_ERR_ARG, "bad dtype %d", dtype);
  if (nfields <= 0 || nfields > SWC_MAX_FIELDS || !fields || !bcs)
    return fail(SWC_ERR_ARG, "bad field list (n=%d)", nfields);
  bool any_prim = false;
  for (int i = 0; i < nfields; ++i) {
    if (!fields[i]) return fail(SWC_ERR_ARG, "field %d is NULL", i);
    if (bcs[i].via_primitive) any_prim = true;
    for (int d = 0; d < 3; ++d)
      for (int s = 0; s < 2; ++s) {
        const SwcBC& b = bcs[i].side[d][s];
        if (b.kind != SWC_BC_PERIODIC && b.kind != SWC_BC_DIRICHLET &&
            b.kind != SWC_BC_NEUMANN && b.kind != SWC_BC_NONE)
          return fail(SWC_ERR_UNSUPPORTED, "Unsupported BC type %d.", b.kind);
        if (b.kind == SWC_BC_DIRICHLET && b.per_layer && !b.planes)
          return fail(SWC_ERR_ARG, "per-layer Dirichlet without planes");
      }
  }
  if (any_prim && (rho_index < 0 || rho_index >= nfields))
    return fail(SWC_ERR_ARG, "primitive BC needs rho (index %d)", rho_index);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int h = grid->halo;
  if (h == 0) return SWC_OK;
  {
    // Every dim periodic for every field, or zero-gradient for every
    // field, no primitive BCs, halos no wider than the interior: one pass
    // instead of three.
    bool all_periodic = !any_prim && h <= grid->nx && h <= grid->ny && h <= grid->nz;
    int clamp[3] = {0, 0, 0};
    for (int d = 0; d < 3 && all_periodic; ++d) {
      int n_per = 0, n_zero = 0;
      for (int i = 0; i < nfields; ++i) {
        const SwcBC& lo = bcs[i].side[d][0];
        const SwcBC& hi = bcs[i].side[d][1];
        if (lo.kind == SWC_BC_PERIODIC || hi.kind == SWC_BC_PERIODIC) ++n_per;
        else if (lo.kind == SWC_BC_NEUMANN && hi.kind == SWC_BC_NEUMANN &&
                 lo.value == 0.0 && hi.value == 0.0 && !lo.per_layer &&
                 !hi.per_layer)
          ++n_zero;
      }
      if (n_per == nfields) clamp[d] = 0;
      else if (n_zero == nfields) clamp[d] = 1;
      else all_periodic = false;
    }
    const long long nxa = grid->nx + 2LL * h, nya = grid->ny + 2LL * h;
    const long long total = 2LL * h * nxa * nya +
                            (long long)grid->nz * (2LL * h * nya + 2LL * h * grid->nx);
    if (all_periodic && total < (1LL << 31)) {
      HaloArgs a;
      memset(&a, 0, sizeof(a));
      a.nf = nfields;
      for (int i = 0; i < nfields; ++i) a.fld[i].f = fields[i];
      a.nx = grid->nx; a.ny = grid->ny; a.nz = grid->nz; a.h = h;
      a.sx = grid->sx; a.sz = grid->sz;
      const int threads = 256;
      const unsigned blocks = (unsigned)((total + threads - 1) / threads);
      if (dtype == SWC_F32)
        halo_periodic_kernel<float><<<blocks, threads, 0, s>>>(
            a, (int)total, clamp[0], clamp[1], clamp[2]);
      else
        halo_periodic_kernel<double><<<blocks, threads, 0, s>>>(
            a, (int)total, clamp[0], clamp[1], clamp[2]);
      note_launch();
      return check_launch("halo_fill");
    }
    // Every side periodic, Dirichlet or Neumann, none on a primitive
    // variable, no periodic dim narrower than the halo: one pass that
    // composes the three (bit for bit the same values).
    bool one_pass = !any_prim && total < (1LL << 31);
    ShellArgs sa;
    memset(&sa, 0, sizeof(sa));
    sa.nf = nfields;
    const int nd[3] = {grid->nx, grid->ny, grid->nz};
    for (int i = 0; i < nfields && one_pass; ++i) {
      sa.fld[i].f = fields[i];
      for (int d = 0; d < 3 && one_pass; ++d) {
        SwcBC lo = bcs[i].side[d][0], hi = bcs[i].side[d][1];
        if (lo.kind == SWC_BC_PERIODIC || hi.kind == SWC_BC_PERIODIC) {
          // A periodic side makes the whole dim periodic (boundary.py:65-68).
          lo.kind = hi.kind = SWC_BC_PERIODIC;
          if (nd[d] < h) one_pass = false;
        } else if (lo.kind == SWC_BC_NONE || hi.kind == SWC_BC_NONE) {
          one_pass = false;
        }
        sa.fld[i].bc[d][0] = lo;
        sa.fld[i].bc[d][1] = hi;
      }
    }
    if (one_pass) {
      sa.nx = grid->nx; sa.ny = grid->ny; sa.nz = grid->nz; sa.h = h;
      sa.sx = grid->sx; sa.sz = grid->sz;
      const int threads = 256;
      const unsigned blocks = (unsigned)((total + threads - 1) / threads);
      if (dtype == SWC_F32)
        halo_shell_kernel<float><<<blocks, threads, 0, s>>>(sa, (int)total);
      else
        halo_shell_kernel<double><<<blocks, threads, 0, s>>>(sa, (int)total);
      note_launch();
      return check_launch("halo_fill");
    }
  }
  // Phase 0: fields with direct BCs; phase 1: fields with primitive BCs,
  // after rho is complete in all three dims.
  for (int phase = 0; phase < (any_prim ? 2 : 1); ++phase) {
    for (int d = 0; d < 3; ++d) {
      HaloArgs a;
      memset(&a, 0, sizeof(a));
      a.dim = d;
      a.nx = grid->nx; a.ny = grid->ny; a.nz = grid->nz; a.h = h;
      a.sx = grid->sx; a.sz = grid->sz;
      a.rho = any_prim ? fields[rho_index] : nullptr;
      for (int i = 0; i < nfields; ++i) {
        if ((bcs[i].via_primitive != 0) != (phase == 1)) continue;
        const SwcBC& lo = bcs[i].side[d][0];
        const SwcBC& hi = bcs[i].side[d][1];
        if (lo.kind == SWC_BC_NONE && hi.kind == SWC_BC_NONE) continue;
        HaloField& hf = a.fld[a.nf++];
        hf.f = fields[i];
        hf.via_prim = bcs[i].via_primitive;
        // A periodic side makes the whole dim periodic (boundary.py:65-68).
        if (lo.kind == SWC_BC_PERIODIC || hi.kind == SWC_BC_PERIODIC) {
          hf.bc[0] = lo; hf.bc[1] = hi;
          hf.bc[0].kind = hf.bc[1].kind = SWC_BC_PERIODIC;
        } else {
          hf.bc[0] = lo; hf.bc[1] = hi;
        }
      }
      if (a.nf == 0) continue;
      const int ext[3] = {grid->nx + 2 * h, grid->ny + 2 * h, grid->nz + 2 * h};
      long long plane = (long long)ext[(d + 1) % 3] * ext[(d + 2) % 3];
      long long total = plane * 2 * a.nf;
      int threads = 256;
      long long blocks = std::min<long long>((total + threads - 1) / threads, 148 * 16);
      if (dtype == SWC_F32)
        halo_kernel<float><<<(unsigned)blocks, threads, 0, s>>>(a);
      else
        halo_kernel<double><<<(unsigned)blocks, threads, 0, s>>>(a);
      note_launch();
      if ((st = check_launch("halo_fill"))) return st;
    }
  }
  return SWC_OK;
}

// SMs of the current device (queried once per device).
static int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
    cached[dev] = n;
  }
  return cached[dev];
}

// Automatic z segment of the stage kernel for `tiles2d` (y, x) tiles and
// `per_sm` resident CTAs per SM. A CTA's time is about (zseg + 1) planes
// (the extra plane: warm-up and the z face below the segment), and the
// launch takes ceil(CTAs / slots) rounds of them, so the segment count that
// minimises rounds x (zseg + 1) is taken: at 256^3 that is 8 segments of 32
// planes (7 rounds of 2048 CTAs on 296 slots) rather than a last round that
// leaves most SMs idle.
static int auto_zseg(long long tiles2d, int nz, int per_sm) {
  const long long slots = (long long)sm_count() * per_sm;
  long long best_cost = -1;
  int best = nz;
  for (int nseg = 1; nseg <= nz; ++nseg) {
    const int zs = (nz + nseg - 1) / nseg;
    if (nseg > 1 && zs == (nz + nseg - 2) / (nseg - 1)) continue;  // same zseg
    if (zs < 4 && nseg > 1) break;
    const long long segs = (nz + zs - 1) / zs;
    const long long rounds = (tiles2d * segs + slots - 1) / slots;
    const long long cost = rounds * (zs + 1);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best = zs;
    }
  }
  return best;
}

// Checks and the kernel arguments shared by swc_rk_stage and
// swc_rk_stage_ext; `nf` conserved fields (5 + scalars); `per_sm` resident
// CTAs per SM and the tile's ty extent (x extent 16) size the z segments.
static int stage_args(const SwcGrid* grid, const SwcScheme* sc, int nf,
                      int per_sm, int ty,
                      const void* const* uk, const void* const* u0,
                      void* const* uout, int32_t mode, double c0, double c1,
                      const double* dt, double* dtmin_out, StageArgs& a) {
  int st = check_grid(grid);
  if (st) return st;
  if (!sc) return fail(SWC_ERR_ARG, "scheme is NULL");
  if (!dtype_ok(sc->dtype)) return fail(SWC_ERR_ARG, "bad dtype %d", sc->dtype);
  if (sc->interp < 0 || sc->interp > 3)
    return fail(SWC_ERR_UNSUPPORTED, "interpolation scheme %d is not implemented", sc->interp);
  if (sc->riemann != SWC_HLL && sc->riemann != SWC_HLLC)
    return fail(SWC_ERR_ARG, "numeric flux scheme %d is not implemented", sc->riemann);
  if (mode < SWC_OUT_RHS || mode > SWC_OUT_AVERAGE)
    return fail(SWC_ERR_ARG, "bad stage mode %d", mode);
  if (!uk || !uout) return fail(SWC_ERR_ARG, "NULL field list");
  for (int v = 0; v < nf; ++v) {
    if (!uk[v] || !uout[v]) return fail(SWC_ERR_ARG, "NULL field %d", v);
    if (uout[v] == uk[v]) return fail(SWC_ERR_ARG, "uout must not alias uk");
    if ((mode == SWC_OUT_CONVEX || mode == SWC_OUT_AVERAGE) && (!u0 || !u0[v]))
      return fail(SWC_ERR_ARG, "stage mode %d needs u0", mode);
  }
  if (mode != SWC_OUT_RHS && !dt) return fail(SWC_ERR_ARG, "dt is NULL");
  const int visc = sc->diffusion ? 1 : 0;
  const int need = stage_halo_needed(sc->interp, visc);
  if (grid->halo < need)
    return fail(SWC_ERR_ARG, "halo_width %d is too small for this scheme (needs %d)",
                grid->halo, need);
  memset(&a, 0, sizeof(a));
  a.nx = grid->nx; a.ny = grid->ny; a.nz = grid->nz; a.halo = grid->halo;
  a.sx = grid->sx; a.sz = grid->sz;
  a.dx = grid->dx; a.dy = grid->dy; a.dz = grid->dz;
  for (int v = 0; v < nf; ++v) {
    a.uk[v] = uk[v];
    a.u0[v] = u0 ? u0[v] : nullptr;
    a.uout[v] = uout[v];
  }
  a.mode = mode; a.c0 = c0; a.c1 = c1; a.dt = dt; a.dtmin_out = dtmin_out;
  for (int d = 0; d < 3; ++d) {
    a.pe[d] = sc->pe_axis[d];
    if (sc->pe_axis[d]) a.has_pe = 1;
    a.g[d] = sc->g[d];
  }
  a.limiter = sc->limiter;
  a.nu = sc->nu; a.pr = sc->pr > 0 ? sc->pr : 1.0;
  a.gravity_mask = sc->gravity_mask;
  int zseg = sc->zseg;
  if (zseg <= 0) {
    const long long tiles2d =
        (long long)((grid->ny + ty - 1) / ty) * ((grid->nx + 15) / 16);
    zseg = auto_zseg(tiles2d, grid->nz, per_sm);
  }
  a.zseg = std::min(zseg, grid->nz);
  return SWC_OK;
}

int swc_rk_stage(const SwcGrid* grid, const SwcScheme* sc,
                 const void* const* uk, const void* const* u0,
                 void* const* uout, int32_t mode, double c0, double c1,
                 const double* dt, double* dtmin_out, void* stream) {
  swc::NvtxRange nvtx_range_("swc_rk_stage");
  if (sc && sc->nscalars != 0)
    return fail(SWC_ERR_UNSUPPORTED,
                "transported scalars go through swc_rk_stage_ext");
  StageArgs a;
  // Resident CTAs per SM of the plain stage kernel (its launch bounds):
  // three for the inviscid single-precision MUSCL stage, two for the other
  // single-precision ones, one in double precision.
  const int per_sm = !sc || sc->dtype != SWC_F32 ? 1
                     : (sc->interp == SWC_MUSCL && !sc->diffusion ? 3 : 2);
  int st = stage_args(grid, sc, 5, per_sm, 16, uk,
                      u0, uout, mode, c0, c1, dt, dtmin_out, a);
  if (st) return st;
  const int visc = sc->diffusion ? 1 : 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int tile = sc->tile;
  int rc;
  if (sc->dtype == SWC_F32) {
    switch (sc->interp) {
      case 0: rc = launch_stage_f32_s0(a, sc->riemann, visc, tile, s); break;
      case 1: rc = launch_stage_f32_s1(a, sc->riemann, visc, tile, s); break;
      case 2: rc = launch_stage_f32_s2(a, sc->riemann, visc, tile, s); break;
      default: rc = launch_stage_f32_s3(a, sc->riemann, visc, tile, s); break;
    }
  } else {
    switch (sc->interp) {
      case 0: rc = launch_stage_f64_s0(a, sc->riemann, visc, tile, s); break;
      case 1: rc = launch_stage_f64_s1(a, sc->riemann, visc, tile, s); break;
      case 2: rc = launch_stage_f64_s2(a, sc->riemann, visc, tile, s); break;
      default: rc = launch_stage_f64_s3(a, sc->riemann, visc, tile, s); break;
    }
  }
  if (rc) return fail(rc, "stage launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return SWC_OK;
}

int swc_rk_stage_ext(const SwcGrid* grid, const SwcScheme* sc,
                     const SwcStageExt* ext, const void* const* uk,
                     const void* const* u0, void* const* uout, int32_t mode,
                     double c0, double c1, const double* dt,
                     double* dtmin_out, void* stream) {
  swc::NvtxRange nvtx_range_("swc_rk_stage_ext");
  if (!sc) return fail(SWC_ERR_ARG, "scheme is NULL");
  const int ns = sc->nscalars;
  if (ns < 0 || ns > 3)
    return fail(SWC_ERR_UNSUPPORTED, "%d transported scalars (at most 3)", ns);
  SwcStageExt e;
  memset(&e, 0, sizeof(e));
  if (ext) {
    e = *ext;
  } else {
    for (int d = 0; d < 3; ++d) e.boundary[d][0] = e.boundary[d][1] = 1;
  }
  if ((e.p_ref == nullptr) != (e.rho_ref == nullptr))
    return fail(SWC_ERR_ARG, "p_ref and rho_ref go together");
  bool any_face = false;
  for (int d = 0; d < 3; ++d)
    for (int sd = 0; sd < 2; ++sd) {
      if (e.nface[d][sd] < 0 || e.nface[d][sd] > SWC_MAX_OVERRIDES ||
          e.nflux[d][sd] < 0 || e.nflux[d][sd] > SWC_MAX_OVERRIDES)
        return fail(SWC_ERR_ARG, "bad override count on side (%d, %d)", d, sd);
      for (int i = 0; i < e.nface[d][sd]; ++i) {
        const SwcOverride& o = e.face[d][sd][i];
        if (o.var == 0)
          return fail(SWC_ERR_UNSUPPORTED,
                      "a density face boundary condition is not supported");
        if (o.var < 1 || o.var > 4 + ns ||
            (o.mode != SWC_FACE_PRIMITIVE && o.mode != SWC_FACE_CONSERVATIVE))
          return fail(SWC_ERR_ARG, "bad face override (var %d, mode %d)", o.var,
                      o.mode);
        any_face = true;
      }
      for (int i = 0; i < e.nflux[d][sd]; ++i) {
        const SwcOverride& o = e.flux[d][sd][i];
        if (o.var < 0 || o.var > 4 + ns || o.mode < SWC_FLUX_CONVECTIVE ||
            o.mode > SWC_FLUX_TOTAL)
          return fail(SWC_ERR_ARG, "bad flux override (var %d, type %d)", o.var,
                      o.mode);
      }
    }
  if (any_face && sc->diffusion)
    return fail(SWC_ERR_UNSUPPORTED,
                "Face boundary conditions are not supported with diffusion "
                "enabled at this time.");
  StageArgs a;
  int st = stage_args(grid, sc, 5 + ns, 1,
                      sc && sc->dtype == SWC_F64 ? 8 : 16, uk, u0, uout, mode,
                      c0, c1, dt, dtmin_out, a);
  if (st) return st;
  const int visc = sc->diffusion ? 1 : 0;
  const int help = e.p_ref ? 1 : 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc;
  if (sc->dtype == SWC_F32) {
    switch (sc->interp) {
      case 0: rc = launch_stage_ext_f32_s0(a, e, sc->riemann, visc, ns, help, s); break;
      case 1: rc = launch_stage_ext_f32_s1(a, e, sc->riemann, visc, ns, help, s); break;
      case 2: rc = launch_stage_ext_f32_s2(a, e, sc->riemann, visc, ns, help, s); break;
      default: rc = launch_stage_ext_f32_s3(a, e, sc->riemann, visc, ns, help, s); break;
    }
  } else {
    switch (sc->interp) {
      case 0: rc = launch_stage_ext_f64_s0(a, e, sc->riemann, visc, ns, help, s); break;
      case 1: rc = launch_stage_ext_f64_s1(a, e, sc->riemann, visc, ns, help, s); break;
      case 2: rc = launch_stage_ext_f64_s2(a, e, sc->riemann, visc, ns, help, s); break;
      default: rc = launch_stage_ext_f64_s3(a, e, sc->riemann, visc, ns, help, s); break;
    }
  }
  if (rc) return fail(rc, "stage launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return SWC_OK;
}

int swc_cfl_reduce(const SwcGrid* grid, const SwcScheme* sc,
                   const void* const* u, double* dtmin_out, void* stream) {
  swc::NvtxRange nvtx_range_("swc_cfl_reduce");
  int st = check_grid(grid);
  if (st) return st;
  if (!sc || !dtype_ok(sc->dtype)) return fail(SWC_ERR_ARG, "bad scheme/dtype");
  if (!u || !dtmin_out) return fail(SWC_ERR_ARG, "NULL argument");
  CflArgs a;
  memset(&a, 0, sizeof(a));
  for (int v = 0; v < 5; ++v) {
    if (!u[v]) return fail(SWC_ERR_ARG, "NULL field %d", v);
    a.u[v] = u[v];
  }
  for (int d = 0; d < 3; ++d) {
    a.pe[d] = sc->pe_axis[d];
    if (sc->pe_axis[d]) a.has_pe = 1;
  }
  a.nx = grid->nx; a.ny = grid->ny; a.nz = grid->nz; a.h = grid->halo;
  a.sx = grid->sx; a.sz = grid->sz;
  a.dx = grid->dx; a.dy = grid->dy; a.dz = grid->dz;
  a.out = dtmin_out;
  long long n = (long long)grid->nx * grid->ny * grid->nz;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (sc->dtype == SWC_F32) cfl_kernel<float><<<blocks_for(n), 256, 0, s>>>(a);
  else cfl_kernel<double><<<blocks_for(n), 256, 0, s>>>(a);
  note_launch();
  return check_launch("cfl_reduce");
}

int swc_clock_begin_step(SwcClock* clock_dev, void* stream) {
  if (!clock_dev) return fail(SWC_ERR_ARG, "clock is NULL");
  clock_begin_kernel<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(clock_dev);
  note_launch();
  return check_launch("clock_begin_step");
}

int swc_clock_end_step(SwcClock* clock_dev, void* stream) {
  if (!clock_dev) return fail(SWC_ERR_ARG, "clock is NULL");
  clock_end_kernel<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(clock_dev);
  note_launch();
  return check_launch("clock_end_step");
}

int swc_clock_status(const SwcClock* clock_dev, void* stream) {
  if (!clock_dev) return fail(SWC_ERR_ARG, "clock is NULL");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  SwcClock c;
  cudaError_t e = cudaMemcpyAsync(&c, clock_dev, sizeof(c), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess)
    return fail(SWC_ERR_LAUNCH, "clock_status: %s", cudaGetErrorString(e));
  if (c.dtmin == 0.0)
    return fail(SWC_ERR_NONFINITE,
                "non-finite or unphysical state (rho, p or rho_e not finite, "
                "or p/rho < 0) after step %lld, t = %.9g",
                (long long)c.step, c.t);
  return SWC_OK;
}

int swc_reconstruct(const SwcGrid* grid, int32_t dtype, int32_t interp,
                    int32_t limiter, int32_t dim, const void* v, void* neg,
                    void* pos, void* stream) {
  int st = check_grid(grid);
  if (st) return st;
  if (!dtype_ok(dtype)) return fail(SWC_ERR_ARG, "bad dtype %d", dtype);
  if (interp < 0 || interp > 3)
    return fail(SWC_ERR_UNSUPPORTED, "interpolation scheme %d is not implemented", interp);
  if (dim < 0 || dim > 2) return fail(SWC_ERR_ARG, "bad dim %d", dim);
  if (!v || !neg || !pos) return fail(SWC_ERR_ARG, "NULL array");
  Geo3 g{grid->nx + 2 * grid->halo, grid->ny + 2 * grid->halo,
         grid->nz + 2 * grid->halo, grid->sx, grid->sz};
  long long n = (long long)g.nxa * g.nya * g.nza;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
#define SWC_RECON(T, S)                                                     \
  recon_kernel<T, S><<<blocks_for(n), 256, 0, s>>>(                         \
      g, dim, limiter, static_cast<const T*>(v), static_cast<T*>(neg),      \
      static_cast<T*>(pos))
  if (dtype == SWC_F32) {
    switch (interp) {
      case 0: SWC_RECON(float, 0); break;
      case 1: SWC_RECON(float, 1); break;
      case 2: SWC_RECON(float, 2); break;
      default: SWC_RECON(float, 3); break;
    }
  } else {
    switch (interp) {
      case 0: SWC_RECON(double, 0); break;
      case 1: SWC_RECON(double, 1); break;
      case 2: SWC_RECON(double, 2); break;
      default: SWC_RECON(double, 3); break;
    }
  }
#undef SWC_RECON
  note_launch();
  return check_launch("reconstruct");
}

static int point_args(int64_t n, int ns, const void* const* ql,
                      const void* const* qr, const void* pe, PointArgs& a) {
  memset(&a, 0, sizeof(a));
  if (n < 0) return fail(SWC_ERR_ARG, "negative size");
  if (ns < 0 || ns > 3)
    return fail(SWC_ERR_UNSUPPORTED, "%d transported scalars (at most 3)", ns);
  if (!ql || !qr) return fail(SWC_ERR_ARG, "NULL state list");
  for (int k = 0; k < 7 + ns; ++k) {
    if (!ql[k] || !qr[k]) return fail(SWC_ERR_ARG, "NULL primitive %d", k);
    a.ql[k] = ql[k];
    a.qr[k] = qr[k];
  }
  a.n = n;
  a.ns = ns;
  a.pe = pe;
  return SWC_OK;
}

int swc_riemann_flux(int64_t n, int32_t dtype, int32_t riemann, int32_t dim,
                     int32_t nscalars, const void* const* prim_neg,
                     const void* const* prim_pos, const void* p_dyn_neg,
                     const void* p_dyn_pos, const void* pe,
                     void* const* flux, void* stream) {
  if (!dtype_ok(dtype)) return fail(SWC_ERR_ARG, "bad dtype %d", dtype);
  if (riemann != SWC_HLL && riemann != SWC_HLLC)
    return fail(SWC_ERR_ARG, "numeric flux scheme %d is not implemented", riemann);
  if (dim < 0 || dim > 2) return fail(SWC_ERR_ARG, "bad dim %d", dim);
  PointArgs a;
  int st = point_args(n, nscalars, prim_neg, prim_pos, pe, a);
  if (st) return st;
  if ((p_dyn_neg == nullptr) != (p_dyn_pos == nullptr))
    return fail(SWC_ERR_ARG, "p_dyn needs both sides");
  a.pdl = p_dyn_neg;
  a.pdr = p_dyn_pos;
  if (!flux) return fail(SWC_ERR_ARG, "NULL flux list");
  for (int k = 0; k < 5 + nscalars; ++k) {
    if (!flux[k]) return fail(SWC_ERR_ARG, "NULL flux %d", k);
    a.out[k] = flux[k];
  }
  if (n == 0) return SWC_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned b = blocks_for(n);
#define SWC_RM(T, RM)                                                        \
  switch (dim) {                                                             \
    case 0: riemann_kernel<T, RM, 0><<<b, 256, 0, s>>>(a); break;           \
    case 1: riemann_kernel<T, RM, 1><<<b, 256, 0, s>>>(a); break;           \
    default: riemann_kernel<T, RM, 2><<<b, 256, 0, s>>>(a); break;          \
  }
  if (dtype == SWC_F32) {
    if (riemann == SWC_HLL) { SWC_RM(float, 0) } else { SWC_RM(float, 1) }
  } else {
    if (riemann == SWC_HLL) { SWC_RM(double, 0) } else { SWC_RM(double, 1) }
  }
#undef SWC_RM
  note_launch();
  return check_launch("riemann_flux");
}

int swc_wave_speeds(int64_t n, int32_t dtype, int32_t dim,
                    const void* const* prim_neg, const void* const* prim_pos,
                    const void* pe, void* s_l, void* s_m, void* s_r,
                    void* stream) {
  if (!dtype_ok(dtype)) return fail(SWC_ERR_ARG, "bad dtype %d", dtype);
  if (dim < 0 || dim > 2) return fail(SWC_ERR_ARG, "bad dim %d", dim);
  PointArgs a;
  int st = point_args(n, 0, prim_neg, prim_pos, pe, a);
  if (st) return st;
  if (!s_l || !s_r) return fail(SWC_ERR_ARG, "NULL output");
  a.sl = s_l; a.sm = s_m; a.sr = s_r;
  if (n == 0) return SWC_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned b = blocks_for(n);
#define SWC_SP(T)                                                            \
  switch (dim) {                                                             \
    case 0: speeds_kernel<T, 0><<<b, 256, 0, s>>>(a); break;                \
    case 1: speeds_kernel<T, 1><<<b, 256, 0, s>>>(a); break;                \
    default: speeds_kernel<T, 2><<<b, 256, 0, s>>>(a); break;               \
  }
  if (dtype == SWC_F32) { SWC_SP(float) } else { SWC_SP(double) }
#undef SWC_SP
  note_launch();
  return check_launch("wave_speeds");
}

int swc_viscous_terms(const SwcGrid* grid, int32_t dtype, int32_t what,
                      const void* const* q, const void* const* rho_face,
                      double nu, double pr, void* const* out, void* stream) {
  int st = check_grid(grid);
  if (st) return st;
  if (!dtype_ok(dtype)) return fail(SWC_ERR_ARG, "bad dtype %d", dtype);
  if (what < SWC_VISC_FLUX || what > SWC_VISC_HEAT)
    return fail(SWC_ERR_ARG, "bad viscous quantity %d", what);
  if (!q || !out) return fail(SWC_ERR_ARG, "NULL argument");
  ViscArgs a;
  memset(&a, 0, sizeof(a));
  a.g = Geo3{grid->nx + 2 * grid->halo, grid->ny + 2 * grid->halo,
             grid->nz + 2 * grid->halo, grid->sx, grid->sz};
  a.what = what;
  // Cell fields each quantity reads: rho and p (FLUX, HEAT), u, v, w (all
  // but HEAT); face densities for STRESS.
  const bool rp = what == SWC_VISC_FLUX || what == SWC_VISC_HEAT;
  const bool vel = what != SWC_VISC_HEAT;
  const bool need[5] = {rp, vel, vel, vel, rp};
  for (int v = 0; v < 5; ++v) {
    if (need[v] && !q[v]) return fail(SWC_ERR_ARG, "NULL cell field %d", v);
    a.q[v] = q[v];
  }
  if (what == SWC_VISC_STRESS) {
    if (!rho_face) return fail(SWC_ERR_ARG, "NULL face densities");
    for (int d = 0; d < 3; ++d) {
      if (!rho_face[d]) return fail(SWC_ERR_ARG, "NULL face density %d", d);
      a.rf[d] = rho_face[d];
    }
  }
  const int nout = what == SWC_VISC_FLUX ? 15 : (what == SWC_VISC_HEAT ? 3 : 9);
  for (int k = 0; k < nout; ++k) {
    if (!out[k]) return fail(SWC_ERR_ARG, "NULL output %d", k);
    a.out[k] = out[k];
  }
  if (rp && !(pr > 0.0)) return fail(SWC_ERR_ARG, "Prandtl number must be > 0");
  a.h[0] = grid->dx; a.h[1] = grid->dy; a.h[2] = grid->dz;
  a.nu = nu;
  a.pr = pr > 0.0 ? pr : 1.0;
  long long n = (long long)a.g.nxa * a.g.nya * a.g.nza;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == SWC_F32) viscous_terms_kernel<float><<<blocks_for(n), 256, 0, s>>>(a);
  else viscous_terms_kernel<double><<<blocks_for(n), 256, 0, s>>>(a);
  note_launch();
  return check_launch("viscous_terms");
}

int swc_stencil(const SwcGrid* grid, int32_t dtype, int32_t op, int32_t dim,
                double h, const void* f, void* out, void* stream) {
  int st = check_grid(grid);
  if (st) return st;
  if (!dtype_ok(dtype)) return fail(SWC_ERR_ARG, "bad dtype %d", dtype);
  if (op < 0 || op > 3) return fail(SWC_ERR_ARG, "bad stencil op %d", op);
  if (dim < 0 || dim > 2)
    return fail(SWC_ERR_ARG, "\"%d\" is not a valid dimension.", dim);
  if (!f || !out || f == out) return fail(SWC_ERR_ARG, "bad arrays");
  Geo3 g{grid->nx + 2 * grid->halo, grid->ny + 2 * grid->halo,
         grid->nz + 2 * grid->halo, grid->sx, grid->sz};
  long long n = (long long)g.nxa * g.nya * g.nza;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == SWC_F32)
    stencil_kernel<float><<<blocks_for(n), 256, 0, s>>>(
        g, op, dim, h, static_cast<const float*>(f), static_cast<float*>(out));
  else
    stencil_kernel<double><<<blocks_for(n), 256, 0, s>>>(
        g, op, dim, h, static_cast<const double*>(f), static_cast<double*>(out));
  note_launch();
  return check_launch("stencil");
}

int swc_rk_combine(int64_t n, int32_t dtype, int32_t mode, double c0,
                   double c1, const double* dt, const void* u0,
                   const void* uk, const void* l, void* out, void* stream) {
  if (!dtype_ok(dtype)) return fail(SWC_ERR_ARG, "bad dtype %d", dtype);
  if (mode != SWC_OUT_EULER && mode != SWC_OUT_CONVEX && mode != SWC_OUT_AVERAGE)
    return fail(SWC_ERR_ARG, "bad combine mode %d", mode);
  if (!dt || !uk || !l || !out || (mode != SWC_OUT_EULER && !u0))
    return fail(SWC_ERR_ARG, "NULL argument");
  if (n <= 0) return n == 0 ? SWC_OK : fail(SWC_ERR_ARG, "negative size");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == SWC_F32)
    combine_kernel<float><<<blocks_for(n), 256, 0, s>>>(
        n, mode, c0, c1, dt, static_cast<const float*>(u0),
        static_cast<const float*>(uk), static_cast<const float*>(l),
        static_cast<float*>(out));
  else
    combine_kernel<double><<<blocks_for(n), 256, 0, s>>>(
        n, mode, c0, c1, dt, static_cast<const double*>(u0),
        static_cast<const double*>(uk), static_cast<const double*>(l),
        static_cast<double*>(out));
  note_launch();
  return check_launch("rk_combine");
}

int swc_rk_step(const SwcGrid* grid, const SwcScheme* scheme,
                const SwcFieldBC* bcs, int32_t order, void* const* u,
                void* const* work, SwcClock* clock_dev, void* stream) {
  swc::NvtxRange nvtx_range_("swc_rk_step");
  int st = check_grid(grid);
  if (st) return st;
  if (!scheme || !bcs || !u || !work || !clock_dev)
    return fail(SWC_ERR_ARG, "NULL argument");
  if (order != 2 && order != 3)
    return fail(SWC_ERR_UNSUPPORTED, "Runge-Kutta order %d is not implemented",
                order);
  for (int v = 0; v < 5; ++v) {
    if (!u[v]) return fail(SWC_ERR_ARG, "NULL field %d", v);
    if (!work[v] || !work[5 + v]) return fail(SWC_ERR_ARG, "NULL work buffer");
  }
  void* w1[5];
  void* w2[5];
  for (int v = 0; v < 5; ++v) {
    w1[v] = work[v];
    w2[v] = work[5 + v];
  }
  const double* dt = &clock_dev->dt;
  double* dtmin = &clock_dev->dtmin;
  if ((st = swc_clock_begin_step(clock_dev, stream))) return st;
  if ((st = swc_halo_fill(grid, scheme->dtype, 5, u, bcs, 0, stream))) return st;
  if ((st = swc_rk_stage(grid, scheme, (const void* const*)u, nullptr, w1,
                         SWC_OUT_EULER, 0.0, 0.0, dt, nullptr, stream)))
    return st;
  if ((st = swc_halo_fill(grid, scheme->dtype, 5, w1, bcs, 0, stream)))
    return st;
  if (order == 3) {
    if ((st = swc_rk_stage(grid, scheme, (const void* const*)w1,
                           (const void* const*)u, w2, SWC_OUT_CONVEX, 0.75,
                           0.25, dt, nullptr, stream)))
      return st;
    if ((st = swc_halo_fill(grid, scheme->dtype, 5, w2, bcs, 0, stream)))
      return st;
    if ((st = swc_rk_stage(grid, scheme, (const void* const*)w2,
                           (const void* const*)u, u, SWC_OUT_CONVEX,
                           1.0 / 3.0, 2.0 / 3.0, dt, dtmin, stream)))
      return st;
  } else {
    if ((st = swc_rk_stage(grid, scheme, (const void* const*)w1,
                           (const void* const*)u, u, SWC_OUT_AVERAGE, 0.5, 0.0,
                           dt, dtmin, stream)))
      return st;
  }
  return swc_clock_end_step(clock_dev, stream);
}

}  // extern "C"
