// swc_rk_step_noalloc: swc_rk_step with its two work states held in a fixed
// array inside this library, for callers that cannot provide device buffers:
// a host that must not allocate device memory once it is running (a plugin
// inside a solver that owns and budgets all device memory up front, a
// real-time loop where an allocation may block or fail) or a binding with no
// way to call a CUDA allocator. Such a caller passes only its state and clock.
//
// The array, g_scratch, is a file-scope __device__ object of
// SWC_NOALLOC_MAX_BYTES bytes; every GPU that loads this library holds it
// until the process exits. Its host-side name is not a device address, so the
// first call on each device looks the address up with cudaGetSymbolAddress
// while that device is current and caches it; that first call should come
// before any stream capture. The cached address belongs to the device's
// primary context of that moment: after cudaDeviceReset (or any other
// teardown of the primary context) it is stale, so this entry point must not
// be called again in that process. The array keeps whatever the last call left in
// it and is shared by all calls, so calls that overlap on the GPU (other
// streams, other host threads on the same device) race on it. Nothing in it
// has to start at zero: the step writes each work state's interior before
// reading it, and the halo fill writes its halos, as with caller buffers
// (except on sides set to SWC_BC_NONE, whose halos keep old contents there
// exactly as they would in a reused caller buffer).
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "swc_launch.h"
#include "swirlc_b200.h"

namespace {

constexpr int kMaxDevices = 64;
constexpr int64_t kWorkFields = 10;  // two RK work states of 5 fields
constexpr int64_t kAlign = 256;

static __device__ __align__(256) unsigned char g_scratch[SWC_NOALLOC_MAX_BYTES];

std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_scratch on the current device, looked up on first use.
int scratch_for_current_device(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return swc::record_error(SWC_ERR_LAUNCH, "rk_step_noalloc: cudaGetDevice: %s",
                             cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return swc::record_error(SWC_ERR_UNSUPPORTED,
                             "rk_step_noalloc: device ordinal %d >= %d", dev,
                             kMaxDevices);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p)
      return swc::record_error(SWC_ERR_LAUNCH,
                               "rk_step_noalloc: cudaGetSymbolAddress: %s",
                               cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return SWC_OK;
}

}  // namespace

extern "C" int swc_rk_step_noalloc(const SwcGrid* grid, const SwcScheme* scheme,
                                   const SwcFieldBC* bcs, int32_t order,
                                   void* const* u, SwcClock* clock_dev,
                                   void* stream) {
  swc::NvtxRange nvtx_range_("swc_rk_step_noalloc");
  if (!grid || !scheme)
    return swc::record_error(SWC_ERR_ARG, "rk_step_noalloc: NULL argument");
  if (scheme->dtype != SWC_F32 && scheme->dtype != SWC_F64)
    return swc::record_error(SWC_ERR_ARG, "rk_step_noalloc: bad dtype %d",
                             scheme->dtype);
  if (grid->nz <= 0 || grid->halo < 0 || grid->sz <= 0)
    return swc::record_error(SWC_ERR_ARG,
                             "rk_step_noalloc: bad grid nz=%d halo=%d sz=%lld",
                             grid->nz, grid->halo, (long long)grid->sz);
  const int64_t elem = scheme->dtype == SWC_F32 ? 4 : 8;
  const int64_t max = (int64_t)SWC_NOALLOC_MAX_BYTES;
  // Elements of one field (halos included); bounded before any product that
  // could overflow.
  const int64_t planes = (int64_t)grid->nz + 2 * (int64_t)grid->halo;
  const int64_t limit_elems = max / (kWorkFields * elem);
  if (grid->sz > limit_elems || planes > limit_elems / grid->sz)
    return swc::record_error(
        SWC_ERR_ARG,
        "rk_step_noalloc: grid needs %g MiB of work space (10 fields of "
        "sz*(nz+2*halo) = %lld*%lld elements of %lld bytes) but the built-in "
        "scratch holds %lld MiB; use swc_rk_step with caller buffers",
        (double)kWorkFields * (double)grid->sz * (double)planes * (double)elem /
            (1024.0 * 1024.0),
        (long long)grid->sz, (long long)planes, (long long)elem,
        (long long)(max >> 20));
  const int64_t field_bytes = grid->sz * planes * elem;
  const int64_t stride = (field_bytes + kAlign - 1) / kAlign * kAlign;
  if (kWorkFields * stride > max)
    return swc::record_error(
        SWC_ERR_ARG,
        "rk_step_noalloc: grid needs %lld bytes of work space after 256-byte "
        "padding but the built-in scratch holds %lld",
        (long long)(kWorkFields * stride), (long long)max);
  void* base = nullptr;
  int st = scratch_for_current_device(&base);
  if (st) return st;
  void* work[kWorkFields];
  for (int64_t i = 0; i < kWorkFields; ++i)
    work[i] = static_cast<unsigned char*>(base) + i * stride;
  return swc_rk_step(grid, scheme, bcs, order, u, work, clock_dev, stream);
}
