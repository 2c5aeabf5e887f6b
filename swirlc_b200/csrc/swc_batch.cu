// swc_batch_step: one time step of many independent grids ("members") with
// a handful of launches for the whole batch. Each RK stage is one batched
// halo pass per dim and one batched stage launch per tile shape; the member
// tables travel in the launch parameters (up to SWC_BATCH_CHUNK members per
// launch), so a step needs no device memory beyond the members' own buffers
// and a CUDA graph captures it whole. Each member keeps its own clock and
// CFL time step.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "swc_halo.cuh"
#include "swc_launch.h"
#include "swirlc_b200.h"

namespace swc {
namespace {

// Kernel parameters are limited to 32764 bytes.
struct HaloBatch {
  int n;
  int bpre[SWC_BATCH_CHUNK + 1];
  HaloMember m[SWC_BATCH_CHUNK];
};
// One-pass halo fill (halo_shell_elem) of up to SWC_BATCH_CHUNK members:
// block b serves member m with bpre[m] <= b < bpre[m+1].
struct ShellMember {
  HaloMember g;
  int clamp[3];
  int total;  // cells of the member's halo shell
};
struct ShellBatch {
  int n;
  int bpre[SWC_BATCH_CHUNK + 1];
  ShellMember m[SWC_BATCH_CHUNK];
};
struct ClockBatch {
  int n;
  SwcClock* c[SWC_BATCH_CHUNK];
};
static_assert(sizeof(HaloBatch) <= 32764, "halo member table too large");
static_assert(sizeof(StageBatch) <= 32764, "stage member table too large");
static_assert(sizeof(ShellBatch) <= 32764, "shell member table too large");
static_assert(sizeof(ClockBatch) <= 32764, "clock table too large");

// Block b serves the member m with bpre[m] <= b < bpre[m+1]; that member's
// blocks stride over its halo elements.
template <typename T>
__global__ void halo_batch_kernel(const HaloBatch b) {
  const int t = blockIdx.x;
  int lo = 0, hi = b.n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (b.bpre[mid] <= t) lo = mid;
    else hi = mid;
  }
  const HaloMember& a = b.m[lo];
  const int nb = b.bpre[lo + 1] - b.bpre[lo];
  const int ext[3] = {a.nx + 2 * a.h, a.ny + 2 * a.h, a.nz + 2 * a.h};
  const long long plane =
      (long long)ext[(a.dim + 1) % 3] * ext[(a.dim + 2) % 3];
  const long long total = plane * 2 * a.nf;
  for (long long i = (long long)(t - b.bpre[lo]) * blockDim.x + threadIdx.x;
       i < total; i += (long long)nb * blockDim.x)
    halo_elem<T>(a, i);
}

template <typename T>
__global__ void shell_batch_kernel(const ShellBatch b) {
  const int t = blockIdx.x;
  int lo = 0, hi = b.n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (b.bpre[mid] <= t) lo = mid;
    else hi = mid;
  }
  const ShellMember& m = b.m[lo];
  const int nb = b.bpre[lo + 1] - b.bpre[lo];
  for (int i = (t - b.bpre[lo]) * blockDim.x + threadIdx.x; i < m.total;
       i += nb * blockDim.x)
    halo_shell_elem<T>(m.g, i, m.clamp[0], m.clamp[1], m.clamp[2]);
}

__global__ void clock_batch_kernel(const ClockBatch b, int end) {
  const int i = threadIdx.x;
  if (i >= b.n) return;
  if (end) clock_end(b.c[i]);
  else clock_begin(b.c[i]);
}

constexpr int kHaloThreads = 256;
constexpr int kHaloMaxBlocksPerMember = 512;

struct Plan {
  const SwcBatchMember* m;
  int tile;  // 1: 16x16, 2: 8x32
  int zseg;
  int ctas;
};

inline void tile_dims(int tile, int& ty, int& tx) {
  ty = tile == 2 ? 8 : 16;
  tx = tile == 2 ? 32 : 16;
}

inline long long tiles2d(const SwcGrid& g, int tile) {
  int ty, tx;
  tile_dims(tile, ty, tx);
  return (long long)((g.ny + ty - 1) / ty) * ((g.nx + tx - 1) / tx);
}

// Field set of a stage: 0 = u, 1 = first work state, 2 = second.
inline void* field_of(const SwcBatchMember& m, int set, int v) {
  return set == 0 ? m.u[v] : m.work[(set - 1) * 5 + v];
}

int check_member(const SwcBatchMember& m, int i, int need) {
  if (check_grid(&m.grid)) return record_error(SWC_ERR_ARG, "member %d: bad grid", i);
  if (m.grid.halo < need)
    return record_error(SWC_ERR_ARG,
                        "member %d: halo_width %d is too small for this scheme "
                        "(needs %d)", i, m.grid.halo, need);
  if (!m.clock) return record_error(SWC_ERR_ARG, "member %d: clock is NULL", i);
  for (int v = 0; v < 5; ++v)
    if (!m.u[v] || !m.work[v] || !m.work[5 + v])
      return record_error(SWC_ERR_ARG, "member %d: NULL field or work buffer", i);
  if (m.tile < 0 || m.tile > 2)
    return record_error(SWC_ERR_ARG, "member %d: bad tile %d", i, m.tile);
  if (m.zseg < 0)
    return record_error(SWC_ERR_ARG, "member %d: bad zseg %d", i, m.zseg);
  for (int v = 0; v < 5; ++v)
    for (int d = 0; d < 3; ++d)
      for (int s = 0; s < 2; ++s) {
        const SwcBC& b = m.bcs[v].side[d][s];
        if (b.kind != SWC_BC_PERIODIC && b.kind != SWC_BC_DIRICHLET &&
            b.kind != SWC_BC_NEUMANN && b.kind != SWC_BC_NONE)
          return record_error(SWC_ERR_UNSUPPORTED, "Unsupported BC type %d.",
                              b.kind);
        if (b.kind == SWC_BC_DIRICHLET && b.per_layer && !b.planes)
          return record_error(SWC_ERR_ARG,
                              "member %d: per-layer Dirichlet without planes", i);
      }
  return SWC_OK;
}

template <typename T>
int launch_shell(const ShellBatch& b, cudaStream_t s) {
  if (b.n == 0) return SWC_OK;
  shell_batch_kernel<T><<<b.bpre[b.n], kHaloThreads, 0, s>>>(b);
  note_launch();
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess
             ? SWC_OK
             : record_error(SWC_ERR_LAUNCH, "batch halo: %s", cudaGetErrorString(e));
}

// Whether member m's halos can be filled in one pass (every dim periodic for
// all 5 fields, or zero-gradient for all of them; no primitive BCs; halos no
// wider than the interior), and with which clamp flags.
bool shell_ok(const SwcBatchMember& m, int clamp[3]) {
  const int h = m.grid.halo;
  if (h <= 0 || h > m.grid.nx || h > m.grid.ny || h > m.grid.nz) return false;
  if (halo_shell_count(m.grid.nx, m.grid.ny, m.grid.nz, h) >= (1LL << 31))
    return false;
  for (int v = 0; v < 5; ++v)
    if (m.bcs[v].via_primitive) return false;
  for (int d = 0; d < 3; ++d) {
    int n_per = 0, n_zero = 0;
    for (int v = 0; v < 5; ++v) {
      const SwcBC& lo = m.bcs[v].side[d][0];
      const SwcBC& hi = m.bcs[v].side[d][1];
      if (lo.kind == SWC_BC_PERIODIC || hi.kind == SWC_BC_PERIODIC) ++n_per;
      else if (lo.kind == SWC_BC_NEUMANN && hi.kind == SWC_BC_NEUMANN &&
               lo.value == 0.0 && hi.value == 0.0 && !lo.per_layer &&
               !hi.per_layer)
        ++n_zero;
    }
    if (n_per == 5) clamp[d] = 0;
    else if (n_zero == 5) clamp[d] = 1;
    else return false;
  }
  return true;
}

template <typename T>
int launch_halo(const HaloBatch& b, cudaStream_t s) {
  if (b.n == 0) return SWC_OK;
  halo_batch_kernel<T><<<b.bpre[b.n], kHaloThreads, 0, s>>>(b);
  note_launch();
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess
             ? SWC_OK
             : record_error(SWC_ERR_LAUNCH, "batch halo: %s", cudaGetErrorString(e));
}

// Halo fill of field set `set` of every member: x, y, z passes of the fields
// with direct BCs, then (if any) of the fields with primitive BCs, as
// swc_halo_fill does for one grid with rho at index 0.
int batch_halo(const std::vector<Plan>& plans, int set, int dtype,
               cudaStream_t s) {
  // Members whose halos take one pass go through shell_batch_kernel; the
  // others through the x, y, z passes below.
  std::vector<char> shell(plans.size(), 0);
  {
    ShellBatch sb;
    memset(&sb, 0, sizeof(sb));
    for (size_t i = 0; i < plans.size(); ++i) {
      const SwcBatchMember& m = *plans[i].m;
      int clamp[3];
      if (!shell_ok(m, clamp)) continue;
      shell[i] = 1;
      ShellMember& sm = sb.m[sb.n];
      memset(&sm, 0, sizeof(sm));
      sm.g.nf = 5;
      for (int v = 0; v < 5; ++v) sm.g.fld[v].f = field_of(m, set, v);
      sm.g.nx = m.grid.nx; sm.g.ny = m.grid.ny; sm.g.nz = m.grid.nz;
      sm.g.h = m.grid.halo;
      sm.g.sx = m.grid.sx; sm.g.sz = m.grid.sz;
      for (int d = 0; d < 3; ++d) sm.clamp[d] = clamp[d];
      sm.total = (int)halo_shell_count(m.grid.nx, m.grid.ny, m.grid.nz, m.grid.halo);
      const int nb = (int)std::min<long long>(
          kHaloMaxBlocksPerMember, (sm.total + kHaloThreads - 1) / kHaloThreads);
      sb.bpre[sb.n + 1] = sb.bpre[sb.n] + nb;
      if (++sb.n == SWC_BATCH_CHUNK) {
        const int rc = dtype == SWC_F32 ? launch_shell<float>(sb, s)
                                        : launch_shell<double>(sb, s);
        if (rc) return rc;
        memset(&sb, 0, sizeof(sb));
      }
    }
    const int rc = dtype == SWC_F32 ? launch_shell<float>(sb, s)
                                    : launch_shell<double>(sb, s);
    if (rc) return rc;
  }
  bool any_prim = false;
  for (const Plan& p : plans)
    for (int v = 0; v < 5; ++v) any_prim |= p.m->bcs[v].via_primitive != 0;
  HaloBatch b;
  for (int phase = 0; phase < (any_prim ? 2 : 1); ++phase) {
    for (int d = 0; d < 3; ++d) {
      memset(&b, 0, sizeof(b));
      for (size_t pi = 0; pi < plans.size(); ++pi) {
        if (shell[pi]) continue;
        const SwcBatchMember& m = *plans[pi].m;
        if (m.grid.halo == 0) continue;
        HaloMember hm;
        memset(&hm, 0, sizeof(hm));
        hm.dim = d;
        hm.nx = m.grid.nx; hm.ny = m.grid.ny; hm.nz = m.grid.nz;
        hm.h = m.grid.halo;
        hm.sx = m.grid.sx; hm.sz = m.grid.sz;
        hm.rho = field_of(m, set, 0);
        for (int v = 0; v < 5; ++v) {
          if ((m.bcs[v].via_primitive != 0) != (phase == 1)) continue;
          const SwcBC& lo = m.bcs[v].side[d][0];
          const SwcBC& hi = m.bcs[v].side[d][1];
          if (lo.kind == SWC_BC_NONE && hi.kind == SWC_BC_NONE) continue;
          HaloField& hf = hm.fld[hm.nf++];
          hf.f = field_of(m, set, v);
          hf.via_prim = m.bcs[v].via_primitive;
          hf.bc[0] = lo;
          hf.bc[1] = hi;
          // A periodic side makes the whole dim periodic (boundary.py:65-68).
          if (lo.kind == SWC_BC_PERIODIC || hi.kind == SWC_BC_PERIODIC)
            hf.bc[0].kind = hf.bc[1].kind = SWC_BC_PERIODIC;
        }
        if (hm.nf == 0) continue;
        const long long ext[3] = {m.grid.nx + 2LL * hm.h, m.grid.ny + 2LL * hm.h,
                                  m.grid.nz + 2LL * hm.h};
        const long long total = ext[(d + 1) % 3] * ext[(d + 2) % 3] * 2 * hm.nf;
        const int nb = (int)std::min<long long>(
            kHaloMaxBlocksPerMember, (total + kHaloThreads - 1) / kHaloThreads);
        b.m[b.n] = hm;
        b.bpre[b.n + 1] = b.bpre[b.n] + nb;
        if (++b.n == SWC_BATCH_CHUNK) {
          const int rc = dtype == SWC_F32 ? launch_halo<float>(b, s)
                                          : launch_halo<double>(b, s);
          if (rc) return rc;
          memset(&b, 0, sizeof(b));
        }
      }
      const int rc = dtype == SWC_F32 ? launch_halo<float>(b, s)
                                      : launch_halo<double>(b, s);
      if (rc) return rc;
    }
  }
  return SWC_OK;
}

// Dynamic shared memory of a batched stage kernel variant.
size_t batch_smem(const SwcScheme* sc, int tile) {
  const int visc = sc->diffusion ? 1 : 0;
  if (sc->dtype == SWC_F32) {
    switch (sc->interp) {
      case 0: return stage_batch_smem_f32_s0(visc, tile);
      case 1: return stage_batch_smem_f32_s1(visc, tile);
      case 2: return stage_batch_smem_f32_s2(visc, tile);
      default: return stage_batch_smem_f32_s3(visc, tile);
    }
  }
  switch (sc->interp) {
    case 0: return stage_batch_smem_f64_s0(visc, tile);
    case 1: return stage_batch_smem_f64_s1(visc, tile);
    case 2: return stage_batch_smem_f64_s2(visc, tile);
    default: return stage_batch_smem_f64_s3(visc, tile);
  }
}

// Shared memory a CTA may use on sm_100 (227 KB), less 1 KB kept for the
// kernel's static shared data.
constexpr size_t kSmemLimit = 227 * 1024 - 1024;

int launch_stage_group(const SwcScheme* sc, const StageBatch& b, int tile,
                       cudaStream_t s) {
  if (b.n == 0) return SWC_OK;
  const int visc = sc->diffusion ? 1 : 0;
  const int nblocks = b.pre[b.n];
  int rc;
  if (sc->dtype == SWC_F32) {
    switch (sc->interp) {
      case 0: rc = launch_stage_batch_f32_s0(b, nblocks, sc->riemann, visc, tile, s); break;
      case 1: rc = launch_stage_batch_f32_s1(b, nblocks, sc->riemann, visc, tile, s); break;
      case 2: rc = launch_stage_batch_f32_s2(b, nblocks, sc->riemann, visc, tile, s); break;
      default: rc = launch_stage_batch_f32_s3(b, nblocks, sc->riemann, visc, tile, s); break;
    }
  } else {
    switch (sc->interp) {
      case 0: rc = launch_stage_batch_f64_s0(b, nblocks, sc->riemann, visc, tile, s); break;
      case 1: rc = launch_stage_batch_f64_s1(b, nblocks, sc->riemann, visc, tile, s); break;
      case 2: rc = launch_stage_batch_f64_s2(b, nblocks, sc->riemann, visc, tile, s); break;
      default: rc = launch_stage_batch_f64_s3(b, nblocks, sc->riemann, visc, tile, s); break;
    }
  }
  if (rc)
    return record_error(rc, "batch stage launch failed: %s",
                        cudaGetErrorString(cudaGetLastError()));
  return SWC_OK;
}

// One fused stage over every member: uk = set `in`, u0 = set 0 (for the
// convex and average modes), out = set `out`; the last stage of a step also
// min-reduces each member's CFL limit into its clock.
int batch_stage(const std::vector<Plan>& plans, const SwcScheme* sc, int in,
                int out, int mode, double c0, double c1, bool reduce,
                cudaStream_t s) {
  StageBatch b;
  for (int tile = 1; tile <= 2; ++tile) {
    memset(&b, 0, sizeof(b));
    for (const Plan& p : plans) {
      if (p.tile != tile) continue;
      const SwcBatchMember& m = *p.m;
      StageArgs& a = b.m[b.n];
      a.nx = m.grid.nx; a.ny = m.grid.ny; a.nz = m.grid.nz; a.halo = m.grid.halo;
      a.sx = m.grid.sx; a.sz = m.grid.sz;
      a.dx = m.grid.dx; a.dy = m.grid.dy; a.dz = m.grid.dz;
      for (int v = 0; v < 5; ++v) {
        a.uk[v] = field_of(m, in, v);
        a.u0[v] = mode >= SWC_OUT_CONVEX ? m.u[v] : nullptr;
        a.uout[v] = field_of(m, out, v);
      }
      a.mode = mode; a.c0 = c0; a.c1 = c1;
      a.dt = &m.clock->dt;
      a.dtmin_out = reduce ? &m.clock->dtmin : nullptr;
      for (int d = 0; d < 3; ++d) {
        a.pe[d] = m.pe_axis[d];
        if (m.pe_axis[d]) a.has_pe = 1;
        a.g[d] = sc->g[d];
      }
      a.limiter = sc->limiter;
      a.nu = sc->nu; a.pr = sc->pr > 0 ? sc->pr : 1.0;
      a.gravity_mask = sc->gravity_mask;
      a.zseg = p.zseg;
      b.pre[b.n + 1] = b.pre[b.n] + p.ctas;
      if (++b.n == SWC_BATCH_CHUNK) {
        const int rc = launch_stage_group(sc, b, tile, s);
        if (rc) return rc;
        memset(&b, 0, sizeof(b));
      }
    }
    const int rc = launch_stage_group(sc, b, tile, s);
    if (rc) return rc;
  }
  return SWC_OK;
}

int batch_clock(const std::vector<Plan>& plans, int end, cudaStream_t s) {
  ClockBatch b;
  memset(&b, 0, sizeof(b));
  size_t i = 0;
  while (i < plans.size()) {
    b.n = 0;
    for (; i < plans.size() && b.n < SWC_BATCH_CHUNK; ++i) b.c[b.n++] = plans[i].m->clock;
    clock_batch_kernel<<<1, SWC_BATCH_CHUNK, 0, s>>>(b, end);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
      return record_error(SWC_ERR_LAUNCH, "batch clock: %s", cudaGetErrorString(e));
  }
  return SWC_OK;
}

}  // namespace
}  // namespace swc

extern "C" int swc_batch_step(const SwcScheme* sc, int32_t order,
                              int32_t nmembers, const SwcBatchMember* members,
                              void* stream) {
  swc::NvtxRange nvtx_range_("swc_batch_step");
  using namespace swc;
  if (!sc) return record_error(SWC_ERR_ARG, "scheme is NULL");
  if (sc->dtype != SWC_F32 && sc->dtype != SWC_F64)
    return record_error(SWC_ERR_ARG, "bad dtype %d", sc->dtype);
  if (sc->interp < 0 || sc->interp > 3)
    return record_error(SWC_ERR_UNSUPPORTED,
                        "interpolation scheme %d is not implemented", sc->interp);
  if (sc->riemann != SWC_HLL && sc->riemann != SWC_HLLC)
    return record_error(SWC_ERR_ARG, "numeric flux scheme %d is not implemented",
                        sc->riemann);
  if (sc->nscalars != 0)
    return record_error(SWC_ERR_UNSUPPORTED,
                        "transported scalars are not supported by the fused stage");
  if (order != 2 && order != 3)
    return record_error(SWC_ERR_UNSUPPORTED,
                        "Runge-Kutta order %d is not implemented", order);
  if (nmembers <= 0 || !members)
    return record_error(SWC_ERR_ARG, "empty member list (n=%d)", nmembers);
  const int need = stage_halo_needed(sc->interp, sc->diffusion ? 1 : 0);
  for (int i = 0; i < nmembers; ++i) {
    const int rc = check_member(members[i], i, need);
    if (rc) return rc;
  }
  // Tiles: 16x16 unless the member asks for 8x32 (which suits members at
  // most 8 cells wide in y, and whose shared-memory layout does not fit for
  // f64 WENO5). The 16x16 instance reproduces swc_rk_step bit for bit; the
  // 8x32 instance of the same arithmetic is scheduled differently by the
  // compiler and can differ from it in the last bit.
  const bool narrow_ok = batch_smem(sc, 2) <= kSmemLimit;
  std::vector<Plan> plans(nmembers);
  for (int i = 0; i < nmembers; ++i) {
    plans[i].m = &members[i];
    if (members[i].tile == 2 && !narrow_ok)
      return record_error(SWC_ERR_UNSUPPORTED,
                          "member %d: tile 8x32 needs %zu bytes of shared "
                          "memory for this scheme and dtype", i,
                          batch_smem(sc, 2));
    plans[i].tile = members[i].tile ? members[i].tile : 1;
  }
  // z planes per CTA for the members that leave it to us: the largest of
  // 64, 32, 16, 8 that still gives about four waves of CTAs (2 per SM on
  // 148 SMs) over the whole batch; longer segments amortise the ring warm-up.
  int zauto = 8;
  for (int z : {64, 32, 16, 8}) {
    long long total = 0;
    for (const Plan& p : plans) {
      const int nz = p.m->grid.nz;
      const int zs = p.m->zseg ? std::min(p.m->zseg, nz) : std::min(z, nz);
      total += tiles2d(p.m->grid, p.tile) * ((nz + zs - 1) / zs);
    }
    if (total >= 4LL * 2 * 148) { zauto = z; break; }
  }
  for (Plan& p : plans) {
    const int nz = p.m->grid.nz;
    p.zseg = std::min(p.m->zseg ? p.m->zseg : zauto, nz);
    const long long ctas = tiles2d(p.m->grid, p.tile) * ((nz + p.zseg - 1) / p.zseg);
    if (ctas > (1LL << 30))
      return record_error(SWC_ERR_ARG, "member grid too large for one launch");
    p.ctas = (int)ctas;
  }
  // Longest CTAs first, so that short ones fill the tail of each launch.
  std::stable_sort(plans.begin(), plans.end(), [](const Plan& x, const Plan& y) {
    return x.zseg > y.zseg;
  });

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int dt = sc->dtype;
  int rc;
  if ((rc = batch_clock(plans, 0, s))) return rc;
  if ((rc = batch_halo(plans, 0, dt, s))) return rc;
  if ((rc = batch_stage(plans, sc, 0, 1, SWC_OUT_EULER, 0.0, 0.0, false, s))) return rc;
  if ((rc = batch_halo(plans, 1, dt, s))) return rc;
  if (order == 3) {
    if ((rc = batch_stage(plans, sc, 1, 2, SWC_OUT_CONVEX, 0.75, 0.25, false, s))) return rc;
    if ((rc = batch_halo(plans, 2, dt, s))) return rc;
    if ((rc = batch_stage(plans, sc, 2, 0, SWC_OUT_CONVEX, 1.0 / 3.0, 2.0 / 3.0, true, s)))
      return rc;
  } else {
    if ((rc = batch_stage(plans, sc, 1, 0, SWC_OUT_AVERAGE, 0.5, 0.0, true, s))) return rc;
  }
  return batch_clock(plans, 1, s);
}
