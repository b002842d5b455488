// Batched RK substep over the boxes of a refinement level.
//
// The reference advances a level box by box: CarpetX launches each scheduled
// routine's loop once per box (AsterX/schedule.ccl:119-228 over the boxes of
// every level), so a level of 512 small boxes costs ~5600 kernel launches per
// substep.  Here every phase of the substep is ONE persistent launch over the
// tiles of all boxes (axb_batch.cuh), the per-box argument blocks live in
// device memory, and the whole substep (12 launches plus one memset of the
// work counters) is stream-ordered and allocation-free, so a caller can
// capture it in a CUDA graph.  The autotuner picks the pencil segment length
// of the y and z flux passes and the number of resident CTAs per SM of the
// persistent grids by timing them on the batch's own boxes.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "axb_batch.cuh"
#include "axb_internal.hxx"
#include "axb_rhs.cuh"

using namespace axb;

namespace axb {
// from the kernel translation units
int batch_rhs_setup(axb_ctx *c, int nbox, const axb_box *boxes, const axb_fields *f,
                    const axb_params *p, const axb_eos *eos, void **out);
int batch_c2p_setup(axb_ctx *c, int nbox, const axb_box *boxes, const axb_fields *f,
                    const axb_params *p, const axb_eos *eos, void **out);
int batch_rk_setup(int nbox, const axb_box *boxes, const axb_fields *f, const axb_fields *fn,
                   int recvar, void **stage_args, void **sync_evolved, void **sync_prims);
uint3 rhs_misc_grid(int which, const axb_box &b);
uint3 flux_grid(int dir, const axb_box &b, int seglen);
uint3 stage_grid(const axb_box &b);
uint3 sync_grid(const axb_box &b, int set);
uint3 c2p_grid(int which, const axb_box &b);
int launch_rhs_misc_batch(int which, const void *args, const TileTable &t,
                          unsigned long long *ctr, int nblocks, cudaStream_t s);
int launch_flux_batch(int recon, int dir, const RhsArgs *args, const TileTable &t,
                      unsigned long long *ctr, const axb_eos &eos, DevStatus *status,
                      int seglen, int nblocks, cudaStream_t s);
int launch_stage_batch(const void *args, const TileTable &t, unsigned long long *ctr,
                       double alpha, double beta, double gdt, int nblocks, cudaStream_t s);
int launch_sync_batch(const void *args, const TileTable &t, unsigned long long *ctr,
                      int nblocks, cudaStream_t s);
int launch_c2p_batch(int which, const void *args, const TileTable &t,
                     unsigned long long *ctr, const axb_eos &eos, DevStatus *status,
                     int nblocks, cudaStream_t s, unsigned long long *queue = nullptr,
                     int deferred_blocks = 0);
bool c2p_batch_fast_ok(int nbox, const axb_box *boxes, const axb_params *p);
} // namespace axb

namespace {

enum Phase {
  P_SOURCES = 0,
  P_FLUX_X,
  P_FLUX_Y,
  P_FLUX_Z,
  P_AUX,
  P_CT,
  P_STAGE,
  P_SYNC_E,
  P_BSTAG,
  P_C2P,
  P_SYNC_P,
  NPHASE
};
const int kRegion[NPHASE] = {AXB_R_SOURCES, AXB_R_FLUX_X, AXB_R_FLUX_Y, AXB_R_FLUX_Z,
                             AXB_R_AUX,     AXB_R_CT,     AXB_R_STAGE,  AXB_R_SYNC,
                             AXB_R_BSTAG,   AXB_R_C2P,    AXB_R_SYNC};
// candidate pencil segments of the y / z flux passes
const int kSeg[] = {8, 16, 32, 64};
constexpr int NSEG = 4;
// candidate persistent-grid sizes, in CTAs per SM
const int kCtas[] = {2, 4, 8, 16};
constexpr int NCTAS = 4;

struct DevTable {
  long long *prefix = nullptr;
  uint3 *grid = nullptr;
  TileTable t{};
};

} // namespace

struct axb_batch {
  int nbox = 0;
  int sms = 148;
  int recon = 0, fd_order = 2;
  const axb_eos *eos = nullptr;
  DevStatus *status = nullptr;
  void *rhs_args = nullptr, *c2p_args = nullptr, *stage_args = nullptr;
  void *sync_e = nullptr, *sync_p = nullptr;
  DevTable tab[NPHASE];
  DevTable flux_seg[2][NSEG]; // y, z tables per candidate segment
  int seg[2] = {2, 2};        // index into kSeg (32)
  int ctas[NPHASE];           // CTAs per SM of each phase's persistent grid
  unsigned long long *ctr = nullptr; // one work counter per phase
  // deferred-cell queue of the recovery's fast pass (null: full cascade)
  unsigned long long *c2p_queue = nullptr;
  long long zones = 0;
};

namespace {

int make_table(const std::vector<axb_box> &boxes, uint3 (*g)(const axb_box &, int), int arg,
               DevTable &out) {
  const int n = int(boxes.size());
  std::vector<long long> prefix(n + 1, 0);
  std::vector<uint3> grid(n);
  for (int b = 0; b < n; ++b) {
    grid[b] = g(boxes[b], arg);
    prefix[b + 1] = prefix[b] + (long long)grid[b].x * grid[b].y * grid[b].z;
  }
  if (cudaMalloc(&out.prefix, (n + 1) * sizeof(long long)) != cudaSuccess ||
      cudaMalloc(&out.grid, n * sizeof(uint3)) != cudaSuccess)
    return AXB_ERR_CUDA;
  if (cudaMemcpy(out.prefix, prefix.data(), (n + 1) * sizeof(long long),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(out.grid, grid.data(), n * sizeof(uint3), cudaMemcpyHostToDevice) !=
          cudaSuccess)
    return AXB_ERR_CUDA;
  out.t.prefix = out.prefix;
  out.t.grid = out.grid;
  out.t.nbox = n;
  out.t.total = prefix[n];
  return AXB_OK;
}

void free_table(DevTable &d) {
  cudaFree(d.prefix);
  cudaFree(d.grid);
  d = DevTable{};
}

uint3 g_sources(const axb_box &b, int) { return rhs_misc_grid(0, b); }
uint3 g_aux(const axb_box &b, int) { return rhs_misc_grid(2, b); }
uint3 g_ct(const axb_box &b, int) { return rhs_misc_grid(3, b); }
uint3 g_flux(const axb_box &b, int dir_seg) { return flux_grid(dir_seg & 3, b, dir_seg >> 2); }
uint3 g_stage(const axb_box &b, int) { return stage_grid(b); }
uint3 g_sync(const axb_box &b, int set) { return sync_grid(b, set); }
uint3 g_c2p(const axb_box &b, int which) { return c2p_grid(which, b); }

int nblocks_for(const axb_batch *B, int phase, long long total) {
  const long long want = (total + BATCH_CHUNK - 1) / BATCH_CHUNK;
  const long long cap = (long long)B->ctas[phase] * B->sms;
  return int(std::max(1LL, std::min(want, cap)));
}

const TileTable &table_of(const axb_batch *B, int phase) {
  if (phase == P_FLUX_Y)
    return B->flux_seg[0][B->seg[0]].t;
  if (phase == P_FLUX_Z)
    return B->flux_seg[1][B->seg[1]].t;
  return B->tab[phase].t;
}

int launch_phase(axb_ctx *c, const axb_batch *B, int phase, double alpha, double beta,
                 double gdt, cudaStream_t s) {
  const TileTable &t = table_of(B, phase);
  const int nb = nblocks_for(B, phase, t.total);
  unsigned long long *ctr = B->ctr + phase;
  axb_mark(c, kRegion[phase], s, true);
  int rc = AXB_OK;
  switch (phase) {
  case P_SOURCES:
    rc = launch_rhs_misc_batch(B->fd_order == 4 ? 1 : 0, B->rhs_args, t, ctr, nb, s);
    break;
  case P_FLUX_X:
  case P_FLUX_Y:
  case P_FLUX_Z: {
    const int dir = phase - P_FLUX_X;
    const int seg = dir == 0 ? 32 : kSeg[B->seg[dir - 1]];
    rc = launch_flux_batch(B->recon, dir, static_cast<const RhsArgs *>(B->rhs_args), t, ctr,
                           *B->eos, B->status, seg, nb, s);
    break;
  }
  case P_AUX: rc = launch_rhs_misc_batch(2, B->rhs_args, t, ctr, nb, s); break;
  case P_CT: rc = launch_rhs_misc_batch(3, B->rhs_args, t, ctr, nb, s); break;
  case P_STAGE: rc = launch_stage_batch(B->stage_args, t, ctr, alpha, beta, gdt, nb, s); break;
  case P_SYNC_E: rc = launch_sync_batch(B->sync_e, t, ctr, nb, s); break;
  case P_BSTAG: rc = launch_c2p_batch(0, B->c2p_args, t, ctr, *B->eos, B->status, nb, s); break;
  case P_C2P:
    rc = launch_c2p_batch(1, B->c2p_args, t, ctr, *B->eos, B->status, nb, s, B->c2p_queue,
                          4 * B->sms);
    break;
  case P_SYNC_P: rc = launch_sync_batch(B->sync_p, t, ctr, nb, s); break;
  }
  axb_mark(c, kRegion[phase], s, false);
  return rc;
}

int run_rhs_phases(axb_ctx *c, const axb_batch *B, cudaStream_t s) {
  for (int ph = P_SOURCES; ph <= P_CT; ++ph) {
    const int rc = launch_phase(c, B, ph, 0, 0, 0, s);
    if (rc)
      return rc;
  }
  return AXB_OK;
}

} // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
AXB_API int axb_batch_destroy(axb_batch *B) {
  if (!B)
    return AXB_ERR_ARG;
  cudaFree(B->rhs_args);
  cudaFree(B->c2p_args);
  cudaFree(B->stage_args);
  cudaFree(B->sync_e);
  cudaFree(B->sync_p);
  cudaFree(B->ctr);
  cudaFree(B->c2p_queue);
  for (auto &t : B->tab)
    free_table(t);
  for (auto &d : B->flux_seg)
    for (auto &t : d)
      free_table(t);
  delete B;
  return AXB_OK;
}

AXB_API int axb_batch_create(axb_ctx *c, int nbox, const axb_box *boxes,
                             const axb_fields *fields, const axb_fields *fields_n,
                             const axb_params *p, const axb_eos *eos, axb_batch **out) {
  if (!c || !boxes || !fields || !fields_n || !p || !eos || !out || nbox < 1)
    return AXB_ERR_ARG;
  *out = nullptr;
  axb_batch *B = new (std::nothrow) axb_batch();
  if (!B)
    return AXB_ERR_ARG;
  B->nbox = nbox;
  B->recon = p->reconstruction_method;
  B->fd_order = p->local_spatial_order;
  B->eos = eos;
  B->status = c->status;
  for (int ph = 0; ph < NPHASE; ++ph)
    B->ctas[ph] = 8;
  cudaDeviceGetAttribute(&B->sms, cudaDevAttrMultiProcessorCount, c->device);
  std::vector<axb_box> bx(boxes, boxes + nbox);
  for (const auto &b : bx)
    B->zones += (long long)b.n[0] * b.n[1] * b.n[2];
  int rc = batch_rhs_setup(c, nbox, boxes, fields, p, eos, &B->rhs_args);
  if (!rc)
    rc = batch_c2p_setup(c, nbox, boxes, fields, p, eos, &B->c2p_args);
  if (!rc)
    rc = batch_rk_setup(nbox, boxes, fields, fields_n, p->recon_type, &B->stage_args,
                        &B->sync_e, &B->sync_p);
  if (!rc)
    rc = make_table(bx, g_sources, 0, B->tab[P_SOURCES]);
  if (!rc)
    rc = make_table(bx, g_flux, 0, B->tab[P_FLUX_X]);
  for (int d = 0; d < 2 && !rc; ++d)
    for (int q = 0; q < NSEG && !rc; ++q)
      rc = make_table(bx, g_flux, (d + 1) | (kSeg[q] << 2), B->flux_seg[d][q]);
  if (!rc)
    rc = make_table(bx, g_aux, 0, B->tab[P_AUX]);
  if (!rc)
    rc = make_table(bx, g_ct, 0, B->tab[P_CT]);
  if (!rc)
    rc = make_table(bx, g_stage, 0, B->tab[P_STAGE]);
  if (!rc)
    rc = make_table(bx, g_sync, 0, B->tab[P_SYNC_E]);
  if (!rc)
    rc = make_table(bx, g_c2p, 0, B->tab[P_BSTAG]);
  if (!rc)
    rc = make_table(bx, g_c2p, 1, B->tab[P_C2P]);
  if (!rc)
    rc = make_table(bx, g_sync,
                    p->recon_type == AXB_RECVAR_Z || p->recon_type == AXB_RECVAR_S ? 2 : 1,
                    B->tab[P_SYNC_P]);
  if (!rc && cudaMalloc(&B->ctr, NPHASE * sizeof(unsigned long long)) != cudaSuccess)
    rc = AXB_ERR_CUDA;
  if (!rc && c2p_batch_fast_ok(nbox, boxes, p) &&
      cudaMalloc(&B->c2p_queue, (B->zones + 1) * sizeof(unsigned long long)) != cudaSuccess)
    rc = AXB_ERR_CUDA;
  if (rc) {
    axb_batch_destroy(B);
    return rc;
  }
  *out = B;
  return AXB_OK;
}

// One RK substep of every box of the batch (as axb_substep does for one box):
// RHS group, stage update, periodic fill of the evolved variables, post-step
// group, periodic fill of the primitives.
AXB_API int axb_batch_substep(axb_ctx *c, axb_batch *B, double alpha, double beta,
                              double gamma, double dt, int periodic, void *stream) {
  if (!c || !B)
    return AXB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  AXB_CUDA_TRY(cudaMemsetAsync(B->ctr, 0, NPHASE * sizeof(unsigned long long), s));
  for (int ph = 0; ph < NPHASE; ++ph) {
    if (!periodic && (ph == P_SYNC_E || ph == P_SYNC_P))
      continue;
    const int rc = launch_phase(c, B, ph, alpha, beta, gamma * dt, s);
    if (rc)
      return rc;
  }
  return AXB_OK;
}

// Autotuner: times the RHS phases on the batch's own boxes for every
// candidate pencil segment of the y and z flux passes and every candidate
// persistent-grid size, and keeps the fastest of each.  The RHS phases
// overwrite what they read back (sources and the x pass write, y and z
// accumulate on top), so repeating them leaves the state as one RHS
// evaluation would; the stage update and the post-step are not touched.
// Synchronous; call it outside any stream capture.  out[0..1] receive the
// chosen y / z segments, out[2] the chosen CTAs per SM of the flux passes.
AXB_API int axb_batch_autotune(axb_ctx *c, axb_batch *B, int *out, void *stream) {
  if (!c || !B)
    return AXB_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  AXB_CUDA_TRY(cudaEventCreate(&e0));
  AXB_CUDA_TRY(cudaEventCreate(&e1));
  const int saved_timing = c->timing;
  c->timing = 0;
  auto time_rhs = [&](int phase, float &ms) -> int {
    AXB_CUDA_TRY(cudaMemsetAsync(B->ctr, 0, NPHASE * sizeof(unsigned long long), s));
    for (int ph = P_SOURCES; ph <= P_CT; ++ph) {
      if (ph == phase)
        AXB_CUDA_TRY(cudaEventRecord(e0, s));
      const int rc = launch_phase(c, B, ph, 0, 0, 0, s);
      if (rc)
        return rc;
      if (ph == phase)
        AXB_CUDA_TRY(cudaEventRecord(e1, s));
    }
    AXB_CUDA_TRY(cudaEventSynchronize(e1));
    AXB_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    return AXB_OK;
  };
  int rc = run_rhs_phases(c, B, s); // warm-up
  // grid size of each RHS phase (segments at their defaults)
  for (int ph = P_SOURCES; ph <= P_CT && !rc; ++ph) {
    int best = B->ctas[ph];
    float best_ms = 1e30f;
    for (int q = 0; q < NCTAS && !rc; ++q) {
      B->ctas[ph] = kCtas[q];
      float ms = 0;
      rc = time_rhs(ph, ms);
      if (!rc && ms < best_ms) {
        best_ms = ms;
        best = kCtas[q];
      }
    }
    B->ctas[ph] = best;
  }
  // segment length of the y and z passes
  for (int d = 0; d < 2 && !rc; ++d) {
    int best = B->seg[d];
    float best_ms = 1e30f;
    for (int q = 0; q < NSEG && !rc; ++q) {
      B->seg[d] = q;
      float ms = 0;
      rc = time_rhs(P_FLUX_Y + d, ms);
      if (!rc && ms < best_ms) {
        best_ms = ms;
        best = q;
      }
    }
    B->seg[d] = best;
  }
  // the post-step and stage phases take the flux passes' grid size
  B->ctas[P_STAGE] = B->ctas[P_SYNC_E] = B->ctas[P_SYNC_P] = B->ctas[P_AUX];
  B->ctas[P_BSTAG] = B->ctas[P_AUX];
  B->ctas[P_C2P] = B->ctas[P_FLUX_Y];
  if (!rc)
    rc = run_rhs_phases(c, B, s); // leave one consistent RHS evaluation behind
  if (!rc && cudaStreamSynchronize(s) != cudaSuccess)
    rc = AXB_ERR_CUDA;
  c->timing = saved_timing;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (out) {
    out[0] = kSeg[B->seg[0]];
    out[1] = kSeg[B->seg[1]];
    out[2] = B->ctas[P_FLUX_Y];
  }
  return rc;
}
