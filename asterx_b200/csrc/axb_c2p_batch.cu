// Batched recovery: the post-step kernels of axb_c2p_box.cuh as persistent
// launches over the tiles of every box of a level (see axb_batch.cuh).
#include "axb_c2p_box.cuh"

using namespace axb;
// ---------------------------------------------------------------------------
// batched forms (see axb_batch.cuh)
// ---------------------------------------------------------------------------
namespace {
__global__ void __launch_bounds__(128) k_bstag_batch(const C2PBoxArgs *args, const TileTable t, unsigned long long *ctr) {
  batch_loop(args, t, ctr, [&](const C2PBoxArgs &a, const uint3 bid) { bstag_body(a, bid); });
}
template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_MINB)
    k_c2p_box_batch(const C2PBoxArgs *args, const TileTable t, unsigned long long *ctr, const EOS eos) {
  batch_loop(args, t, ctr, [&](const C2PBoxArgs &a, const uint3 bid) {
    c2p_box_body<EOS>(a, eos, bid);
  });
}
template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_FAST_MINB)
    k_c2p_fast_batch(const C2PBoxArgs *args, const TileTable t, unsigned long long *ctr,
                     const EOS eos, const C2PQueue q) {
  batch_loop(args, t, ctr, [&](const C2PBoxArgs &a, const uint3 bid, int box) {
    c2p_fast_body<EOS>(a, eos, bid, box, q);
  });
}
template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_MINB)
    k_c2p_deferred_batch(const C2PBoxArgs *args, const EOS eos, const C2PQueue q) {
  c2p_deferred_body([&](int box) -> const C2PBoxArgs & { return args[box]; }, eos, q);
}
template <class EOS>
int launch_c2p_batch_eos(const C2PBoxArgs *a, const TileTable &t, unsigned long long *ctr,
                         const EOS &eos, int nblocks, unsigned long long *queue,
                         int deferred_blocks, cudaStream_t s) {
  if (!queue) {
    k_c2p_box_batch<<<nblocks, 128, 0, s>>>(a, t, ctr, eos);
  } else {
    C2PQueue q;
    q.count = queue;
    q.cell = queue + 1;
    if (cudaMemsetAsync(q.count, 0, sizeof(unsigned long long), s) != cudaSuccess)
      return AXB_ERR_CUDA;
    k_c2p_fast_batch<<<nblocks, 128, 0, s>>>(a, t, ctr, eos, q);
    k_c2p_deferred_batch<<<deferred_blocks, 128, 0, s>>>(a, eos, q);
  }
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}
} // namespace

namespace axb {
// The per-box post-step argument blocks of a batch (checked as
// axb_con2prim_group checks them), in device memory.
int batch_c2p_setup(axb_ctx *c, int nbox, const axb_box *boxes, const axb_fields *f,
                    const axb_params *p, const axb_eos *eos, void **out) {
  *out = nullptr;
  C2PBoxArgs *h = new (std::nothrow) C2PBoxArgs[nbox];
  if (!h)
    return AXB_ERR_ARG;
  for (int b = 0; b < nbox; ++b) {
    int rc = fill_c2p_args(c, boxes + b, f + b, p, eos, h[b]);
    if (!rc && p->use_uct)
      rc = AXB_ERR_UNSUPPORTED; // the batched RHS is flux CT only
    h[b].b.packed = 1;
    if (rc) {
      delete[] h;
      return rc;
    }
  }
  int rc = AXB_OK;
  if (cudaMalloc(out, nbox * sizeof(C2PBoxArgs)) != cudaSuccess ||
      cudaMemcpy(*out, h, nbox * sizeof(C2PBoxArgs), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = AXB_ERR_CUDA;
  delete[] h;
  return rc;
}

// batched grids over packed (i, j) planes: face curl (0), recovery (1)
uint3 c2p_grid(int which, const axb_box &b) {
  const int T = 128;
  const int e = which == 0 ? 2 : 0;
  const long long plane = (long long)(b.n[0] + e) * (b.n[1] + e);
  return make_uint3(unsigned((plane + T - 1) / T), 1, b.n[2] + e);
}

// `queue` (count, then room for every interior cell of the batch) selects
// the fast pass + deferred full cascade (Palenzuela first), else the full
// cascade in one launch.
int launch_c2p_batch(int which, const void *args, const TileTable &t,
                     unsigned long long *ctr, const axb_eos &eos, DevStatus *status,
                     int nblocks, cudaStream_t s, unsigned long long *queue,
                     int deferred_blocks) {
  if (t.total == 0)
    return AXB_OK;
  const C2PBoxArgs *a = static_cast<const C2PBoxArgs *>(args);
  if (which == 0) {
    k_bstag_batch<<<nblocks, 128, 0, s>>>(a, t, ctr);
    return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
  }
  if (eos.kind == 1)
    return launch_c2p_batch_eos(a, t, ctr, tab_for_launch(eos, status), nblocks, queue,
                                deferred_blocks, s);
  return launch_c2p_batch_eos(a, t, ctr, eos.ideal, nblocks, queue, deferred_blocks, s);
}

// whether a batch can take the fast pass: Palenzuela first, boxes and
// extents within the queue's packing
bool c2p_batch_fast_ok(int nbox, const axb_box *boxes, const axb_params *p) {
  if (p->c2p_prime != AXB_C2P_PALENZUELA || nbox > C2P_QUEUE_MAX_BOXES)
    return false;
  for (int b = 0; b < nbox; ++b)
    if (!c2p_queue_fits(boxes[b]))
      return false;
  return true;
}
} // namespace axb

