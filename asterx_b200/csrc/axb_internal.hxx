// Host-side internals shared by the translation units of the engine.
#pragma once

#include <cuda_runtime.h>

#include "axb_common.cuh"
#include "axb_eos.cuh"

struct axb_ctx {
  int device;
  axb::DevStatus *status; // device
  axb::DevStatus *status_host_pinned;
  char last_error[256];
};

// Tabulated-EOS device data (see axb_tab.cuh); declared here so the host
// handle can own it.
namespace axb {
struct EosTab;
}

struct axb_eos {
  int kind; // 0 ideal gas, 1 tabulated
  axb::EosIdeal ideal;
  axb::EosPoly poly;
  axb::EosTab *tab_host; // host copy of the device descriptor (tabulated)
  double *tab_dev;       // device table storage
};

namespace axb {
// launchers (one per translation unit of kernels)
int launch_flux_pass(int dir, int recon, const struct RhsArgs &a,
                     const axb_eos &eos, int seglen, cudaStream_t s);
int launch_rhs_misc(int which, const struct RhsArgs &a, cudaStream_t s);
} // namespace axb

#define AXB_CUDA_TRY(call)                                                     \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess)                                                     \
      return AXB_ERR_CUDA;                                                     \
  } while (0)
