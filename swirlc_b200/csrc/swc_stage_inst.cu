// Instantiates the fused stage kernel for one (dtype, scheme) pair; compiled
// once per pair with -DSWC_T=<float|double> -DSWC_SCHEME=<0..3>
// -DSWC_SUFFIX=<name> so the 32 kernel variants build in parallel.
#include "swc_launch.h"

#ifndef SWC_T
#error "SWC_T must be defined"
#endif

#ifndef SWC_MULTI_TILE
#define SWC_MULTI_TILE 0
#endif

#define SWC_CAT2(a, b) a##b
#define SWC_CAT(a, b) SWC_CAT2(a, b)

namespace swc {
namespace {

// Tile shapes (TY along y, TX along x); 256 threads each.
template <typename T, int RM, bool V, int TY, int TX>
int launch_tile(const StageArgs& a, cudaStream_t st) {
  using Lay = Layout<T, SWC_SCHEME, V, TY, TX>;
  auto kern = stage_kernel<T, SWC_SCHEME, RM, V, TY, TX>;
  // Set once per process (before any graph capture: the first launch of a
  // variant is always eager).
  static int attr_set = 0;
  cudaError_t e;
  if (!attr_set) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Lay::SMEM);
    if (e != cudaSuccess) return SWC_ERR_LAUNCH;
    attr_set = 1;
  }
  dim3 grid((a.ny + TY - 1) / TY, (a.nx + TX - 1) / TX,
            (a.nz + a.zseg - 1) / a.zseg);
  kern<<<grid, TY * TX, Lay::SMEM, st>>>(a);
  note_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SWC_OK : SWC_ERR_LAUNCH;
}

template <typename T, int RM, bool V>
int launch_rm(const StageArgs& a, int tile, cudaStream_t st) {
#if SWC_MULTI_TILE
  switch (tile) {
    case 1: return launch_tile<T, RM, V, 16, 16>(a, st);
    case 2: return launch_tile<T, RM, V, 8, 32>(a, st);
    default: return launch_tile<T, RM, V, 32, 8>(a, st);
  }
#else
  (void)tile;
  return launch_tile<T, RM, V, 16, 16>(a, st);
#endif
}

// Batched launch of `nblocks` CTAs over the members of `b`. Tiles: 1 = 16x16
// (y x x), 2 = 8x32 for members with ny <= 8.
template <typename T, int RM, bool V, int TY, int TX>
int launch_batch_tile(const StageBatch& b, int nblocks, cudaStream_t st) {
  using Lay = Layout<T, SWC_SCHEME, V, TY, TX>;
  auto kern = stage_batch_kernel<T, SWC_SCHEME, RM, V, TY, TX>;
  static int attr_set = 0;
  cudaError_t e;
  if (!attr_set) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)Lay::SMEM);
    if (e != cudaSuccess) return SWC_ERR_LAUNCH;
    attr_set = 1;
  }
  kern<<<nblocks, TY * TX, Lay::SMEM, st>>>(b);
  note_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SWC_OK : SWC_ERR_LAUNCH;
}

template <typename T, int RM, bool V>
int launch_batch_rm(const StageBatch& b, int nblocks, int tile,
                    cudaStream_t st) {
  if (tile == 2) return launch_batch_tile<T, RM, V, 8, 32>(b, nblocks, st);
  return launch_batch_tile<T, RM, V, 16, 16>(b, nblocks, st);
}

// Extended stage (scalars, helper states, face/flux overrides): 16x16 tiles
// in f32, 8x16 in f64 so that the larger ring fits in shared memory.
template <typename T, int RM, bool V, int NS, bool HELP>
int launch_ext_v(const StageArgs& a, const SwcStageExt& e, cudaStream_t st) {
  constexpr int TY = sizeof(T) == 4 ? 16 : 8, TX = 16;
  using Lay = Layout<T, SWC_SCHEME, V, TY, TX, NS, HELP>;
  auto kern = stage_kernel_ext<T, SWC_SCHEME, RM, V, TY, TX, NS, HELP>;
  static int attr_set = 0;
  cudaError_t err;
  if (!attr_set) {
    err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)Lay::SMEM);
    if (err != cudaSuccess) return SWC_ERR_LAUNCH;
    attr_set = 1;
  }
  dim3 grid((a.ny + TY - 1) / TY, (a.nx + TX - 1) / TX,
            (a.nz + a.zseg - 1) / a.zseg);
  kern<<<grid, TY * TX, Lay::SMEM, st>>>(a, e);
  note_launch();
  err = cudaGetLastError();
  return err == cudaSuccess ? SWC_OK : SWC_ERR_LAUNCH;
}

template <typename T, int RM, bool V>
int launch_ext_rm(const StageArgs& a, const SwcStageExt& e, int ns, bool help,
                  cudaStream_t st) {
  switch (ns * 2 + (help ? 1 : 0)) {
    case 0: return launch_ext_v<T, RM, V, 0, false>(a, e, st);
    case 1: return launch_ext_v<T, RM, V, 0, true>(a, e, st);
    case 2: return launch_ext_v<T, RM, V, 1, false>(a, e, st);
    case 3: return launch_ext_v<T, RM, V, 1, true>(a, e, st);
    case 4: return launch_ext_v<T, RM, V, 2, false>(a, e, st);
    case 5: return launch_ext_v<T, RM, V, 2, true>(a, e, st);
    case 6: return launch_ext_v<T, RM, V, 3, false>(a, e, st);
    default: return launch_ext_v<T, RM, V, 3, true>(a, e, st);
  }
}

template <typename T, bool V>
size_t smem_tile(int tile) {
#if SWC_MULTI_TILE
  switch (tile) {
    case 1: return Layout<T, SWC_SCHEME, V, 16, 16>::SMEM;
    case 2: return Layout<T, SWC_SCHEME, V, 8, 32>::SMEM;
    default: return Layout<T, SWC_SCHEME, V, 32, 8>::SMEM;
  }
#else
  (void)tile;
  return Layout<T, SWC_SCHEME, V, 16, 16>::SMEM;
#endif
}

}  // namespace

int SWC_CAT(launch_stage_, SWC_SUFFIX)(const StageArgs& a, int riemann,
                                       int visc, int tile, cudaStream_t st) {
  using T = SWC_T;
  if (riemann == SWC_HLL)
    return visc ? launch_rm<T, 0, true>(a, tile, st)
                : launch_rm<T, 0, false>(a, tile, st);
  return visc ? launch_rm<T, 1, true>(a, tile, st)
              : launch_rm<T, 1, false>(a, tile, st);
}

int SWC_CAT(launch_stage_batch_, SWC_SUFFIX)(const StageBatch& b, int nblocks,
                                             int riemann, int visc, int tile,
                                             cudaStream_t st) {
  using T = SWC_T;
  if (riemann == SWC_HLL)
    return visc ? launch_batch_rm<T, 0, true>(b, nblocks, tile, st)
                : launch_batch_rm<T, 0, false>(b, nblocks, tile, st);
  return visc ? launch_batch_rm<T, 1, true>(b, nblocks, tile, st)
              : launch_batch_rm<T, 1, false>(b, nblocks, tile, st);
}

int SWC_CAT(launch_stage_ext_, SWC_SUFFIX)(const StageArgs& a,
                                           const SwcStageExt& e, int riemann,
                                           int visc, int ns, int help,
                                           cudaStream_t st) {
  using T = SWC_T;
  const bool hp = help != 0;
  if (riemann == SWC_HLL)
    return visc ? launch_ext_rm<T, 0, true>(a, e, ns, hp, st)
                : launch_ext_rm<T, 0, false>(a, e, ns, hp, st);
  return visc ? launch_ext_rm<T, 1, true>(a, e, ns, hp, st)
              : launch_ext_rm<T, 1, false>(a, e, ns, hp, st);
}

size_t SWC_CAT(stage_batch_smem_, SWC_SUFFIX)(int visc, int tile) {
  using T = SWC_T;
  if (tile == 2)
    return visc ? Layout<T, SWC_SCHEME, true, 8, 32>::SMEM
                : Layout<T, SWC_SCHEME, false, 8, 32>::SMEM;
  return visc ? Layout<T, SWC_SCHEME, true, 16, 16>::SMEM
              : Layout<T, SWC_SCHEME, false, 16, 16>::SMEM;
}

size_t SWC_CAT(stage_smem_, SWC_SUFFIX)(int visc, int tile) {
  using T = SWC_T;
  return visc ? smem_tile<T, true>(tile) : smem_tile<T, false>(tile);
}

}  // namespace swc
