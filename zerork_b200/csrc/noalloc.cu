// noalloc.cu -- rates + Jacobian entry point that allocates no device memory.
//
// zrk_rates_jac_dev gives the global-workspace mapping of the rates kernel a
// scratch buffer that the library cudaMallocs on first use.  Some callers
// cannot let a library allocate while they run: a CFD code that hands the
// whole GPU to its own pool allocator at start-up (and fails any allocation
// made behind the pool's back), a solver stepping inside a region where a
// cudaMalloc would synchronize the device and stall its other streams, or a
// host that must keep its device memory footprint fixed after set-up.
// zrk_rates_jac_dev_noalloc runs the same kernel with its workspace in the
// file-scope array below, so the call itself allocates nothing.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/zerork_b200.h"
#include "capi_internal.h"

namespace zrk {
namespace {

// 8 MiB of per-CTA workspace slices, held by every device that loads the
// library until the process exits.
constexpr size_t kNoAllocScratchBytes = ZRK_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (host code only
// sees a host-side stand-in under that name).  Looked up once per device.
int scratch_address(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return set_error(ZRK_ERR_NO_DEVICE, "device index out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_scratch_ptr[dev] = static_cast<double *>(p);
  }
  *out = g_scratch_ptr[dev];
  return ZRK_OK;
}

}  // namespace
}  // namespace zrk

using namespace zrk;

extern "C" int zrk_rates_jac_dev_noalloc(zrk_mech_t m, int n, int ld, const double *T, const double *P,
                                         const double *Y, double *wdot, double *jac, double *ydot,
                                         void *stream) {
  if (!m) return set_error(ZRK_ERR_INVALID_HANDLE, "null handle");
  if (n < 0 || ld < n) return set_error(ZRK_ERR_INVALID_ARGUMENT, "need 0 <= n <= ld");
  if (n == 0) return ZRK_OK;
  if (!T || !P || !Y || !wdot) return set_error(ZRK_ERR_INVALID_POINTER, "null array");
  MechHandle *h = reinterpret_cast<MechHandle *>(m);
  if (!h->dev) return set_error(ZRK_ERR_NO_DEVICE, "handle has no device tables (zrk_mech_parse)");
  const DevMech &dm = h->dev->view();
  // the handle's tile mapping, always with the workspace in global memory
  LaunchCfg cfg = h->cfg;
  cfg.global_ws = true;
  const size_t slice = rates_jac_ws_bytes(dm, cfg);
  const size_t fit = kNoAllocScratchBytes / slice;
  if (fit == 0)
    return set_error(ZRK_ERR_INVALID_ARGUMENT,
                     "no-alloc scratch too small: one tile of this mechanism needs " +
                         std::to_string(slice) + " bytes, the fixed array holds " +
                         std::to_string(kNoAllocScratchBytes) + " (choose a smaller tile with "
                         "zrk_mech_set_launch or use zrk_rates_jac_dev)");
  const int ntiles = (n + cfg.ts - 1) / cfg.ts;
  int grid = cfg.grid > 0 ? cfg.grid : ntiles;
  if (grid > ntiles) grid = ntiles;
  if ((size_t)grid > fit) grid = (int)fit;  // tiles beyond the grid are taken in turn
  cfg.grid = grid;
  double *scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != ZRK_OK) return rc;
  RatesJacArgs a;
  a.n = n;
  a.ld = ld;
  a.T = T;
  a.P = P;
  a.Y = Y;
  a.wdot = wdot;
  a.jac = jac;
  a.ydot = ydot;
  a.scratch = scratch;
  a.scratch_bytes = kNoAllocScratchBytes;
  KinParams kp{h->Tref, h->mmf, h->lim, std::sqrt(2.2204460492503131e-16)};
  cudaError_t e = launch_rates_jac(dm, a, kp, cfg, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_error(e, "rates_jac launch (no-alloc)");
  return ZRK_OK;
}
