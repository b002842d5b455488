// Runge-Kutta stage update of the evolved variables and the periodic ghost
// fill of one box (the single-box form of the driver's SYNC).
#include <cstring>

#include "axb_internal.hxx"

using namespace axb;

namespace {

constexpr int NEVOLVED = 11;
// evolved grid functions and their centring (1 = cell-centred along x,y,z)
const int kEvolved[NEVOLVED] = {AXB_GF_dens, AXB_GF_momx, AXB_GF_momy, AXB_GF_momz,
                                AXB_GF_tau,  AXB_GF_DYe,  AXB_GF_DEnt, AXB_GF_Avec_x,
                                AXB_GF_Avec_y, AXB_GF_Avec_z, AXB_GF_Psi};
const int kEvolvedRhs[NEVOLVED] = {
    AXB_GF_densrhs, AXB_GF_momxrhs, AXB_GF_momyrhs, AXB_GF_momzrhs,
    AXB_GF_taurhs,  AXB_GF_DYe_rhs, AXB_GF_DEntrhs, AXB_GF_Avec_x_rhs,
    AXB_GF_Avec_y_rhs, AXB_GF_Avec_z_rhs, AXB_GF_Psi_rhs};
const int kCent[NEVOLVED][3] = {{1, 1, 1}, {1, 1, 1}, {1, 1, 1}, {1, 1, 1},
                                {1, 1, 1}, {1, 1, 1}, {1, 1, 1}, {1, 0, 0},
                                {0, 1, 0}, {0, 0, 1}, {0, 0, 0}};

struct StageArgs {
  BoxDev b;
  double *out[NEVOLVED];
  const double *un[NEVOLVED], *uk[NEVOLVED], *rhs[NEVOLVED];
  int cent[NEVOLVED][3];
  double alpha, beta, gdt;
};

// U_out = alpha U_n + beta U_k + (gamma dt) RHS on the interior of each
// field's centring (cells for hydro, edges for A, vertices for Psi).
__global__ void __launch_bounds__(128) k_rk_stage(const StageArgs a) {
  const BoxDev &b = a.b;
  const int i = b.ng + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = b.ng + blockIdx.y;
  const int k = b.ng + blockIdx.z;
  if (i > b.ng + b.n[0])
    return;
  const long long I = b.at(i, j, k);
  const int ijk[3] = {i, j, k};
#pragma unroll
  for (int v = 0; v < NEVOLVED; ++v) {
    bool in = true;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      in &= ijk[d] < b.ng + b.n[d] + (a.cent[v][d] ? 0 : 1);
    if (in)
      a.out[v][I] = a.alpha * a.un[v][I] + a.beta * a.uk[v][I] + a.gdt * a.rhs[v][I];
  }
}

struct SyncArgs {
  BoxDev b;
  double *f[AXB_NUM_GF];
  int cent[AXB_NUM_GF][3];
  int nf;
};

AXB_D int wrap(int i, int ng, int n) {
  int r = (i - ng) % n;
  if (r < 0)
    r += n;
  return ng + r;
}

// Periodic ghost fill: every point outside the interior of its centring
// takes the value of its periodic image inside the interior.  One block
// handles one (j, k) row of one field.
__global__ void __launch_bounds__(128) k_sync_periodic(const SyncArgs a) {
  const BoxDev &b = a.b;
  const int v = blockIdx.z;
  const int j = blockIdx.x;
  const int k = blockIdx.y;
  double *f = a.f[v];
  const int *c = a.cent[v];
  const int ng = b.ng;
  const int hi[3] = {ng + b.n[0] + (c[0] ? 0 : 1), ng + b.n[1] + (c[1] ? 0 : 1),
                     ng + b.n[2] + (c[2] ? 0 : 1)};
  const int npts0 = b.n[0] + 2 * ng + (c[0] ? 0 : 1);
  const bool row_in = j >= ng && j < hi[1] && k >= ng && k < hi[2];
  const int js = (j >= ng && j < hi[1]) ? j : wrap(j, ng, b.n[1]);
  const int ks = (k >= ng && k < hi[2]) ? k : wrap(k, ng, b.n[2]);
  if (j >= b.n[1] + 2 * ng + (c[1] ? 0 : 1) || k >= b.n[2] + 2 * ng + (c[2] ? 0 : 1))
    return;
  for (int i = threadIdx.x; i < npts0; i += blockDim.x) {
    const bool i_in = i >= ng && i < hi[0];
    if (row_in && i_in)
      continue;
    const int is = i_in ? i : wrap(i, ng, b.n[0]);
    f[b.at(i, j, k)] = f[b.at(is, js, ks)];
  }
}

int centring_of(int gf, int c[3]) {
  c[0] = c[1] = c[2] = 1; // cell
  switch (gf) {
  case AXB_GF_Avec_x: case AXB_GF_Avec_x_rhs: c[1] = c[2] = 0; break;
  case AXB_GF_Avec_y: case AXB_GF_Avec_y_rhs: c[0] = c[2] = 0; break;
  case AXB_GF_Avec_z: case AXB_GF_Avec_z_rhs: c[0] = c[1] = 0; break;
  case AXB_GF_dBx_stag: c[0] = 0; break;
  case AXB_GF_dBy_stag: c[1] = 0; break;
  case AXB_GF_dBz_stag: c[2] = 0; break;
  default:
    if ((gf >= AXB_GF_gxx && gf <= AXB_GF_kzz) || gf == AXB_GF_Psi ||
        gf == AXB_GF_Psi_rhs || (gf >= AXB_GF_Fx && gf <= AXB_GF_G))
      c[0] = c[1] = c[2] = 0;
  }
  return 0;
}

} // namespace

// One Runge-Kutta stage of the 11 evolved variables (dens, mom, tau, DYe,
// DEnt, Avec, Psi) on the interior:
//   out = alpha * U_n + beta * U_k + gamma * dt * RHS
// (the stage combine of CarpetX's ODESolvers, which the reference's
// scheduled routines rely on; SSP-RK3 in Shu-Osher form uses
// (alpha, beta, gamma) = (0,1,1), (3/4,1/4,1/4), (1/3,2/3,2/3)).
// `out`, `un` and `uk` may alias; the RHS is read from `rhs`.
AXB_API int axb_rk_stage(axb_ctx *c, const axb_box *box, const axb_fields *out,
                         const axb_fields *un, const axb_fields *uk,
                         const axb_fields *rhs, double alpha, double beta,
                         double gamma, double dt, void *stream) {
  if (!c || !box || !out || !un || !uk || !rhs)
    return AXB_ERR_ARG;
  StageArgs a;
  a.b = make_box(*box);
  for (int v = 0; v < NEVOLVED; ++v) {
    a.out[v] = out->gf[kEvolved[v]];
    a.un[v] = un->gf[kEvolved[v]];
    a.uk[v] = uk->gf[kEvolved[v]];
    a.rhs[v] = rhs->gf[kEvolvedRhs[v]];
    if (!a.out[v] || !a.un[v] || !a.uk[v] || !a.rhs[v])
      return AXB_ERR_ARG;
    for (int d = 0; d < 3; ++d)
      a.cent[v][d] = kCent[v][d];
  }
  a.alpha = alpha;
  a.beta = beta;
  a.gdt = gamma * dt;
  const int T = 128;
  const dim3 grid((box->n[0] + 1 + T - 1) / T, box->n[1] + 1, box->n[2] + 1);
  axb_mark(c, AXB_R_STAGE, (cudaStream_t)stream, true);
  k_rk_stage<<<grid, T, 0, (cudaStream_t)stream>>>(a);
  axb_mark(c, AXB_R_STAGE, (cudaStream_t)stream, false);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

// Periodic ghost fill of the grid functions listed in `ids` (each with its
// own centring) on one box: the single-box stand-in for the driver's SYNC
// with periodic outer boundaries.
AXB_API int axb_sync_periodic(axb_ctx *c, const axb_box *box,
                              const axb_fields *f, const int *ids, int nids,
                              void *stream) {
  if (!c || !box || !f || !ids || nids < 1 || nids > AXB_NUM_GF)
    return AXB_ERR_ARG;
  if (box->ng < 1)
    return AXB_ERR_GHOSTS;
  for (int d = 0; d < 3; ++d)
    if (box->n[d] < box->ng)
      return AXB_ERR_ARG; // a ghost layer must fit inside one period
  SyncArgs a;
  a.b = make_box(*box);
  a.nf = nids;
  for (int q = 0; q < nids; ++q) {
    if (ids[q] < 0 || ids[q] >= AXB_NUM_GF || !f->gf[ids[q]])
      return AXB_ERR_ARG;
    a.f[q] = f->gf[ids[q]];
    centring_of(ids[q], a.cent[q]);
  }
  const dim3 grid(box->n[1] + 2 * box->ng + 1, box->n[2] + 2 * box->ng + 1, nids);
  axb_mark(c, AXB_R_SYNC, (cudaStream_t)stream, true);
  k_sync_periodic<<<grid, 128, 0, (cudaStream_t)stream>>>(a);
  axb_mark(c, AXB_R_SYNC, (cudaStream_t)stream, false);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}
