// Host-side declarations shared by the C-ABI translation unit and the
// per-(dtype, scheme) stage-kernel instantiation units.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "swc_stage.cuh"

namespace swc {

// A named NVTX range over one C-ABI call, so that profilers show the
// library's steps, stages, halo fills and adjoint stages on the host
// timeline (NVTX v3 is header-only; with no tool attached a push and pop
// cost a few nanoseconds).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Launches the fused stage kernel for one (dtype, scheme); returns 0 or a
// negative SWC status. Defined in swc_stage_inst.cu, compiled once per pair.
#define SWC_DECL_STAGE(SUFFIX)                                               \
  int launch_stage_##SUFFIX(const StageArgs& a, int riemann, int visc,       \
                            int tile, cudaStream_t st);                      \
  int launch_stage_batch_##SUFFIX(const StageBatch& b, int nblocks,          \
                                  int riemann, int visc, int tile,           \
                                  cudaStream_t st);                          \
  int launch_stage_ext_##SUFFIX(const StageArgs& a, const SwcStageExt& e,   \
                                int riemann, int visc, int ns, int help,     \
                                cudaStream_t st);                            \
  size_t stage_smem_##SUFFIX(int visc, int tile);                          \
  size_t stage_batch_smem_##SUFFIX(int visc, int tile);
SWC_DECL_STAGE(f32_s0)
SWC_DECL_STAGE(f32_s1)
SWC_DECL_STAGE(f32_s2)
SWC_DECL_STAGE(f32_s3)
SWC_DECL_STAGE(f64_s0)
SWC_DECL_STAGE(f64_s1)
SWC_DECL_STAGE(f64_s2)
SWC_DECL_STAGE(f64_s3)
#undef SWC_DECL_STAGE

// Halo layers the stage kernel needs for a scheme.
inline int stage_halo_needed(int scheme, int visc) {
  switch (scheme) {
    case 0: return visc ? Geom<0, true>::NEED : Geom<0, false>::NEED;
    case 1: return visc ? Geom<1, true>::NEED : Geom<1, false>::NEED;
    case 2: return visc ? Geom<2, true>::NEED : Geom<2, false>::NEED;
    default: return visc ? Geom<3, true>::NEED : Geom<3, false>::NEED;
  }
}

// Counts kernel launches issued by this library (thread-local).
void note_launch(int n = 1);

// Sets the message swc_last_error() reports on this thread; returns `code`.
int record_error(int code, const char* fmt, ...);

// SWC_OK, or SWC_ERR_ARG with the message set, for a grid's sizes/strides.
int check_grid(const SwcGrid* g);

// Device clock updates (SwcClock): start and end of a time step.
__device__ __forceinline__ void clock_begin(SwcClock* c) {
  if (c->cfl > 0.0) {
    double dt = c->cfl * c->dtmin;
    if (c->t_end > 0.0) dt = fmin(dt, c->t_end - c->t);
    c->dt = dt;
  }
  c->dtmin = 1e300;
}
__device__ __forceinline__ void clock_end(SwcClock* c) {
  c->t += c->dt;
  c->step += 1;
}

}  // namespace swc
