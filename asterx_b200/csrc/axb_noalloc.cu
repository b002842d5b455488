// Allocation-free form of the RHS group.
//
// Some callers cannot allocate device memory at all: code that runs inside a
// host framework whose memory manager owns every device allocation, tools
// that are not allowed to call cudaMalloc on a device they share, or drivers
// that must not grow their footprint after set-up.  They cannot provide the
// 20 scratch grid functions that axb_rhs_group needs (partial divergences,
// face B fluxes, vertex auxiliaries).  axb_rhs_group_noalloc takes the same
// inputs and outputs but keeps that scratch, and the status block, in
// file-scope device arrays of this library: every GPU that loads the library
// holds these 16 MiB until the process exits.
#include <cstring>
#include <mutex>

#include "axb_internal.hxx"

extern "C" int axb_rhs_group(axb_ctx *, const axb_box *, const axb_fields *,
                             const axb_params *, const axb_eos *, void *);

namespace {

constexpr size_t kScratchDoubles = size_t(1) << 21; // 16 MiB of FP64
constexpr int kNScratch = 20;
constexpr int kMaxDevices = 64;

// In host code these names are host-side stand-ins, not device addresses;
// their device addresses come from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];
static __device__ __align__(256) axb::DevStatus g_noalloc_status;

const int kScratchIds[kNScratch] = {
    AXB_GF_acc_dens, AXB_GF_acc_momx, AXB_GF_acc_momy, AXB_GF_acc_momz,
    AXB_GF_acc_tau,  AXB_GF_acc_DYe,  AXB_GF_acc_DEnt, AXB_GF_fxBy,
    AXB_GF_fxBz,     AXB_GF_fyBx,     AXB_GF_fyBz,     AXB_GF_fzBx,
    AXB_GF_fzBy,     AXB_GF_Fx,       AXB_GF_Fy,       AXB_GF_Fz,
    AXB_GF_Fbetax,   AXB_GF_Fbetay,   AXB_GF_Fbetaz,   AXB_GF_G};

std::mutex g_mu;
double *g_scratch_dev[kMaxDevices];
axb::DevStatus *g_status_dev[kMaxDevices];

// Device addresses of the two arrays on the current device, looked up once
// per device with that device current.
int device_arrays(int dev, double **scratch, axb::DevStatus **status) {
  if (dev < 0 || dev >= kMaxDevices)
    return AXB_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_dev[dev]) {
    void *p = nullptr, *q = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess ||
        cudaGetSymbolAddress(&q, g_noalloc_status) != cudaSuccess)
      return AXB_ERR_CUDA;
    g_scratch_dev[dev] = static_cast<double *>(p);
    g_status_dev[dev] = static_cast<axb::DevStatus *>(q);
  }
  *scratch = g_scratch_dev[dev];
  *status = g_status_dev[dev];
  return AXB_OK;
}

} // namespace

// axb_rhs_group without caller-provided scratch and without a context.
// See include/asterx_b200.h for the contract.
AXB_API int axb_rhs_group_noalloc(const axb_box *box, const axb_fields *fields,
                                  const axb_params *params, const axb_eos *eos,
                                  void *stream) {
  if (!box || !fields || !params || !eos)
    return AXB_ERR_ARG;
  // sizes are range-checked before any arithmetic on them (axb_rhs_group
  // checks the box again in full)
  constexpr int64_t kMaxExtent = int64_t(1) << 15;
  for (int d = 0; d < 3; ++d)
    if (box->n[d] < 1 || box->n[d] > kMaxExtent)
      return AXB_ERR_ARG;
  if (box->ng < 0 || box->ng > kMaxExtent || box->sy < 1 || box->sz < 1)
    return AXB_ERR_ARG;
  if (box->sz > (int64_t)kScratchDoubles)
    return AXB_ERR_TOO_LARGE;
  // one scratch grid function = the box's whole index space, rounded up to
  // 32 doubles so every slice starts on a 256-byte boundary
  const size_t planes = (size_t)box->n[2] + 2 * (size_t)box->ng + 1;
  const size_t per = ((size_t)box->sz * planes + 31) / 32 * 32;
  if (per > kScratchDoubles / kNScratch)
    return AXB_ERR_TOO_LARGE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess)
    return AXB_ERR_NO_DEVICE;
  double *scratch = nullptr;
  axb::DevStatus *status = nullptr;
  int rc = device_arrays(dev, &scratch, &status);
  if (rc)
    return rc;
  axb_fields f = *fields;
  for (int q = 0; q < kNScratch; ++q)
    f.gf[kScratchIds[q]] = scratch + q * per;
  // the status block accumulates (error bits, CFL maximum): start from zero
  if (cudaMemsetAsync(status, 0, sizeof(axb::DevStatus), (cudaStream_t)stream) !=
      cudaSuccess)
    return AXB_ERR_CUDA;
  axb_ctx ctx{};
  ctx.device = dev;
  ctx.status = status;
  ctx.timing = 0;
  return axb_rhs_group(&ctx, box, &f, params, eos, stream);
}
