// Host-side internals shared by the translation units of the engine.
#pragma once

#include <cuda_runtime.h>

#include "axb_common.cuh"
#include "axb_eos.cuh"
#include "axb_tab.cuh"

// Kernel regions timed by the optional per-launch CUDA events.
enum axb_region {
  AXB_R_SOURCES = 0,
  AXB_R_FLUX_X,
  AXB_R_FLUX_Y,
  AXB_R_FLUX_Z,
  AXB_R_AUX,
  AXB_R_CT,
  AXB_R_STAGE,
  AXB_R_SYNC,
  AXB_R_BSTAG,
  AXB_R_C2P,
  AXB_R_C2P_CELLS,
  AXB_R_MLP,
  AXB_R_TMUNU,
  AXB_R_ERROR,
  AXB_NREGIONS
};
constexpr int AXB_EVENT_POOL = 4096;

struct axb_ctx {
  int device;
  axb::DevStatus *status; // device
  axb::DevStatus *status_host_pinned;
  char last_error[256];
  // per-launch timing (off unless axb_timing_begin was called)
  int timing = 0;
  int ev_used = 0;
  cudaEvent_t *ev = nullptr; // 2 * AXB_EVENT_POOL
  int *ev_region = nullptr;
  // stream-ordered pool of per-call scratch (the recovery's deferred-cell
  // queue); keeps its memory between calls
  cudaMemPool_t pool = nullptr;
  // a second stream for the RHS group's kernels that do not depend on the
  // flux passes (sources, vertex auxiliaries), forked from and joined back
  // into the caller's stream with events; created on first use, in
  // contexts from axb_ctx_create only (which destroys them)
  int allow_side = 0;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_sources = nullptr, ev_aux = nullptr;
};

// Stream-ordered scratch: from the context's pool, or (during a stream
// capture) from the device's default pool, which captures as a graph
// allocation node.  Release with cudaFreeAsync on the same stream.
inline cudaError_t axb_scratch_alloc(axb_ctx *c, void **p, size_t bytes, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess)
    return cudaErrorUnknown;
  if (cs != cudaStreamCaptureStatusNone)
    return cudaMallocAsync(p, bytes, s);
  if (!c->pool) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = c->device;
    cudaError_t e = cudaMemPoolCreate(&c->pool, &props);
    if (e != cudaSuccess) {
      c->pool = nullptr;
      return e;
    }
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  return cudaMallocFromPoolAsync(p, bytes, c->pool, s);
}

// Record the start / end event of one timed launch (no-ops unless timing).
inline void axb_mark(axb_ctx *c, int region, cudaStream_t s, bool start) {
  if (!c || !c->timing)
    return;
  if (start) {
    if (c->ev_used >= AXB_EVENT_POOL)
      return;
    c->ev_region[c->ev_used] = region;
    cudaEventRecord(c->ev[2 * c->ev_used], s);
  } else {
    if (c->ev_used >= AXB_EVENT_POOL)
      return;
    cudaEventRecord(c->ev[2 * c->ev_used + 1], s);
    ++c->ev_used;
  }
}

struct axb_eos {
  int kind; // 0 ideal gas, 1 tabulated
  axb::EosIdeal ideal;
  axb::EosPoly poly;
  // tabulated: the same descriptor over host memory (host-side atmosphere
  // set-up) and over device memory (kernels); each owns one allocation
  axb::EosTab tab_h, tab_d;
  double *tab_host; // axes + compact table, host
  double *tab_dev;  // axes + compact table, device
};

// The device descriptor of a tabulated EOS with its root-cap flag pointed at
// the context's status word.
inline axb::EosTab tab_for_launch(const axb_eos &e, axb::DevStatus *st) {
  axb::EosTab t = e.tab_d;
  t.err = st ? &st->error_word : nullptr;
  return t;
}

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
