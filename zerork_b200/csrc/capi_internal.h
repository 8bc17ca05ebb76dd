// capi_internal.h -- handle type shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "devmech.h"
#include "kinetics.h"
#include "mech.h"

namespace zrk {

struct MechHandle {
  MechTables tables;
  JacPattern pattern;
  std::unique_ptr<DeviceMechanism> dev;
  LaunchCfg cfg;
  double Tref = 1.0, mmf = 1.0e-30, lim = 1.0e22;
  void *scratch = nullptr;
  size_t scratch_bytes = 0;
  std::vector<void *> host_bufs;
  void *pipe = nullptr;  // host-entry pipeline slots (device)
  size_t pipe_bytes = 0;
  cudaStream_t pipe_stream[2] = {nullptr, nullptr};
  ~MechHandle();
  cudaError_t ensure_scratch(size_t bytes);
  cudaError_t ensure_pipe(size_t bytes);
};

int set_error(int code, const std::string &msg);
int cuda_error(cudaError_t e, const char *what);
LaunchCfg default_launch(const DevMech &m);

}  // namespace zrk
