// Runge-Kutta stage update of the evolved variables and the periodic ghost
// fill of one box (the single-box form of the driver's SYNC).
#include <algorithm>
#include <cstring>
#include <vector>

#include "axb_batch.cuh"
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
AXB_D void rk_stage_body(const StageArgs &a, double alpha, double beta, double gdt,
                         const uint3 bid) {
  const BoxDev &b = a.b;
  int i, j;
  const int k = b.ng + bid.z;
  if (!b.row_ij(b.ng, b.n[0] + 1, b.ng, b.n[1] + 1, bid, i, j))
    return;
  const long long I = b.at(i, j, k);
  const int ijk[3] = {i, j, k};
#pragma unroll
  for (int v = 0; v < NEVOLVED; ++v) {
    bool in = true;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      in &= ijk[d] < b.ng + b.n[d] + (a.cent[v][d] ? 0 : 1);
    // explicit rounding order, the same as the stage update fused into the
    // z flux pass and the CT kernel (stage_combine)
    if (in)
      a.out[v][I] = fma(gdt, a.rhs[v][I], fma(beta, a.uk[v][I], alpha * a.un[v][I]));
  }
}
__global__ void __launch_bounds__(128)
    k_rk_stage(const StageArgs a) {
  rk_stage_body(a, a.alpha, a.beta, a.gdt, blockIdx);
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
// takes the value of its periodic image inside the interior.  One thread per
// ghost point, enumerated slab below, slab above, then the ghost rows and
// row ends of the middle planes, so no thread idles on interior points.
struct Shell {
  long long A, B, Cm, G;
  int N[3], hi[3], ng;
  AXB_HD Shell(const BoxDev &b, const int c[3]) {
    ng = b.ng;
    for (int d = 0; d < 3; ++d) {
      N[d] = b.n[d] + 2 * ng + (c[d] ? 0 : 1);
      hi[d] = ng + b.n[d] + (c[d] ? 0 : 1);
    }
    const long long plane = (long long)N[0] * N[1];
    A = ng * plane;
    B = (long long)(N[2] - hi[2]) * plane;
    Cm = (long long)(ng + N[1] - hi[1]) * N[0] + (long long)(hi[1] - ng) * (ng + N[0] - hi[0]);
    G = A + B + (long long)(hi[2] - ng) * Cm;
  }
  AXB_HD void point(long long g, int &i, int &j, int &k) const {
    const long long plane = (long long)N[0] * N[1];
    if (g < A + B) {
      k = g < A ? int(g / plane) : hi[2] + int((g - A) / plane);
      const long long r = g < A ? g % plane : (g - A) % plane;
      j = int(r / N[0]);
      i = int(r % N[0]);
      return;
    }
    g -= A + B;
    k = ng + int(g / Cm);
    long long r = g % Cm;
    const long long lowrows = (long long)ng * N[0], highrows = (long long)(N[1] - hi[1]) * N[0];
    if (r < lowrows) {
      j = int(r / N[0]);
      i = int(r % N[0]);
    } else if (r < lowrows + highrows) {
      r -= lowrows;
      j = hi[1] + int(r / N[0]);
      i = int(r % N[0]);
    } else {
      r -= lowrows + highrows;
      const int per = ng + N[0] - hi[0];
      j = ng + int(r / per);
      const int q = int(r % per);
      i = q < ng ? q : hi[0] + (q - ng);
    }
  }
};

AXB_D void sync_shell_body(const SyncArgs &a, const uint3 bid) {
  const BoxDev &b = a.b;
  const int v = bid.z;
  const Shell sh(b, a.cent[v]);
  const long long g = (long long)bid.x * blockDim.x + threadIdx.x;
  if (g >= sh.G)
    return;
  int i, j, k;
  sh.point(g, i, j, k);
  const int ng = b.ng;
  const int is = (i >= ng && i < sh.hi[0]) ? i : wrap(i, ng, b.n[0]);
  const int js = (j >= ng && j < sh.hi[1]) ? j : wrap(j, ng, b.n[1]);
  const int ks = (k >= ng && k < sh.hi[2]) ? k : wrap(k, ng, b.n[2]);
  double *f = a.f[v];
  f[b.at(i, j, k)] = f[b.at(is, js, ks)];
}

__global__ void __launch_bounds__(128) k_sync_shell(const SyncArgs a) {
  sync_shell_body(a, blockIdx);
}

int centring_of(int gf, int c[3]) {
  c[0] = c[1] = c[2] = 1; // cell
  switch (gf) {
  case AXB_GF_Avec_x: case AXB_GF_Avec_x_rhs: c[1] = c[2] = 0; break;
  case AXB_GF_Avec_y: case AXB_GF_Avec_y_rhs: c[0] = c[2] = 0; break;
  case AXB_GF_Avec_z: case AXB_GF_Avec_z_rhs: c[0] = c[1] = 0; break;
  case AXB_GF_dBx_stag: case AXB_GF_fxBy: case AXB_GF_fxBz:
  case AXB_GF_vtilde_y_xface: case AXB_GF_vtilde_z_xface:
  case AXB_GF_amax_xface: case AXB_GF_amin_xface: c[0] = 0; break;
  case AXB_GF_dBy_stag: case AXB_GF_fyBx: case AXB_GF_fyBz:
  case AXB_GF_vtilde_z_yface: case AXB_GF_vtilde_x_yface:
  case AXB_GF_amax_yface: case AXB_GF_amin_yface: c[1] = 0; break;
  case AXB_GF_dBz_stag: case AXB_GF_fzBx: case AXB_GF_fzBy:
  case AXB_GF_vtilde_x_zface: case AXB_GF_vtilde_y_zface:
  case AXB_GF_amax_zface: case AXB_GF_amin_zface: c[2] = 0; break;
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
  // one thread per ghost point of the largest centring among the fields
  long long gmax = 0;
  for (int q = 0; q < nids; ++q)
    gmax = std::max(gmax, Shell(a.b, a.cent[q]).G);
  const dim3 grid(unsigned((gmax + 127) / 128), 1, nids);
  axb_mark(c, AXB_R_SYNC, (cudaStream_t)stream, true);
  k_sync_shell<<<grid, 128, 0, (cudaStream_t)stream>>>(a);
  axb_mark(c, AXB_R_SYNC, (cudaStream_t)stream, false);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// batched forms (see axb_batch.cuh)
// ---------------------------------------------------------------------------
namespace {

__global__ void __launch_bounds__(128)
    k_rk_stage_batch(const StageArgs *args, const TileTable t, unsigned long long *ctr, double alpha, double beta,
                     double gdt) {
  batch_loop(args, t, ctr, [&](const StageArgs &a, const uint3 bid) {
    rk_stage_body(a, alpha, beta, gdt, bid);
  });
}

__global__ void __launch_bounds__(128)
    k_sync_batch(const SyncArgs *args, const TileTable t, unsigned long long *ctr) {
  batch_loop(args, t, ctr, [&](const SyncArgs &a, const uint3 bid) { sync_shell_body(a, bid); });
}

template <class T> int upload(const std::vector<T> &h, void **out) {
  *out = nullptr;
  if (h.empty())
    return AXB_OK;
  if (cudaMalloc(out, h.size() * sizeof(T)) != cudaSuccess)
    return AXB_ERR_CUDA;
  if (cudaMemcpy(*out, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return AXB_ERR_CUDA;
  return AXB_OK;
}

} // namespace

namespace axb {

// Per-box stage and ghost-fill argument blocks of a batch, in device memory.
int batch_rk_setup(int nbox, const axb_box *boxes, const axb_fields *f, const axb_fields *fn,
                   int recvar, void **stage_args, void **sync_evolved, void **sync_prims) {
  // the 12 cell-centred primitives, plus the reconstructed zvec or svec
  // when the fluxes reconstruct one of those instead of the velocity
  int prims[15] = {AXB_GF_rho,   AXB_GF_velx, AXB_GF_vely,        AXB_GF_velz,
                   AXB_GF_eps,   AXB_GF_press, AXB_GF_temperature, AXB_GF_Ye,
                   AXB_GF_entropy, AXB_GF_Bvecx, AXB_GF_Bvecy,     AXB_GF_Bvecz};
  int nprims = 12;
  if (recvar == AXB_RECVAR_Z || recvar == AXB_RECVAR_S) {
    const int first = recvar == AXB_RECVAR_Z ? AXB_GF_zvec_x : AXB_GF_svec_x;
    for (int q = 0; q < 3; ++q)
      prims[nprims++] = first + q;
  }
  std::vector<StageArgs> st(nbox);
  std::vector<SyncArgs> se(nbox), sp(nbox);
  for (int b = 0; b < nbox; ++b) {
    const axb_box &box = boxes[b];
    if (box.ng < 1)
      return AXB_ERR_GHOSTS;
    for (int d = 0; d < 3; ++d)
      if (box.n[d] < box.ng)
        return AXB_ERR_ARG;
    StageArgs &a = st[b];
    std::memset(&a, 0, sizeof a);
    a.b = make_box(box);
    a.b.packed = 1;
    for (int v = 0; v < NEVOLVED; ++v) {
      a.out[v] = f[b].gf[kEvolved[v]];
      a.un[v] = fn[b].gf[kEvolved[v]];
      a.uk[v] = f[b].gf[kEvolved[v]];
      a.rhs[v] = f[b].gf[kEvolvedRhs[v]];
      if (!a.out[v] || !a.un[v] || !a.rhs[v])
        return AXB_ERR_ARG;
      for (int d = 0; d < 3; ++d)
        a.cent[v][d] = kCent[v][d];
    }
    for (int pass = 0; pass < 2; ++pass) {
      SyncArgs &y = pass ? sp[b] : se[b];
      std::memset(&y, 0, sizeof y);
      y.b = make_box(box);
      const int nf = pass ? nprims : NEVOLVED;
      y.nf = nf;
      for (int q = 0; q < nf; ++q) {
        const int id = pass ? prims[q] : kEvolved[q];
        y.f[q] = f[b].gf[id];
        if (!y.f[q])
          return AXB_ERR_ARG;
        centring_of(id, y.cent[q]);
      }
    }
  }
  int rc = upload(st, stage_args);
  if (!rc)
    rc = upload(se, sync_evolved);
  if (!rc)
    rc = upload(sp, sync_prims);
  return rc;
}

// batched grids: the stage update over packed (i, j) planes, and the ghost
// fill over the ghost points of the largest centring of the set (0: the 11
// evolved variables, 1: the 12 cell-centred primitives)
uint3 stage_grid(const axb_box &b) {
  const long long plane = (long long)(b.n[0] + 1) * (b.n[1] + 1);
  return make_uint3(unsigned((plane + 127) / 128), 1, b.n[2] + 1);
}
// set 0: the 11 evolved variables; 1: the 12 cell-centred primitives; 2: the
// primitives and the reconstructed zvec or svec (15 cell-centred fields)
uint3 sync_grid(const axb_box &b, int set) {
  const BoxDev bd = make_box(b);
  long long g = 0;
  const int nf = set == 0 ? NEVOLVED : set == 1 ? 12 : 15;
  for (int q = 0; q < nf; ++q) {
    int c[3] = {1, 1, 1};
    if (!set)
      for (int d = 0; d < 3; ++d)
        c[d] = kCent[q][d];
    const Shell sh(bd, c);
    g = std::max(g, sh.G);
  }
  return make_uint3(unsigned((g + 127) / 128), 1, nf);
}

int launch_stage_batch(const void *args, const TileTable &t, unsigned long long *ctr,
                       double alpha, double beta, double gdt, int nblocks, cudaStream_t s) {
  if (t.total == 0)
    return AXB_OK;
  k_rk_stage_batch<<<nblocks, 128, 0, s>>>(static_cast<const StageArgs *>(args), t, ctr,
                                           alpha, beta, gdt);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

int launch_sync_batch(const void *args, const TileTable &t, unsigned long long *ctr,
                      int nblocks, cudaStream_t s) {
  if (t.total == 0)
    return AXB_OK;
  k_sync_batch<<<nblocks, 128, 0, s>>>(static_cast<const SyncArgs *>(args), t, ctr);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

} // namespace axb

namespace axb {
// The centring of a grid function (1 = cell-centred along x, y, z), for the
// other translation units of the library.
int gf_centring(int gf, int c[3]) { return centring_of(gf, c); }
} // namespace axb
