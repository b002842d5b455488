// Outer-boundary fill and the general Runge-Kutta combination of the evolved
// variables: the pieces of CarpetX's ODESolvers and boundary handling that
// the reference's scheduled routines run inside (no counterpart in the
// reference sources), for multi-step evolutions of one box with physical
// outer boundaries.
#include <algorithm>

#include "axb_internal.hxx"

using namespace axb;

namespace axb {
int gf_centring(int gf, int c[3]); // axb_rk.cu
}

namespace {

constexpr int NEVOLVED = 11;
const int kEvolvedIds[NEVOLVED] = {AXB_GF_dens, AXB_GF_momx, AXB_GF_momy, AXB_GF_momz,
                                   AXB_GF_tau,  AXB_GF_DYe,  AXB_GF_DEnt, AXB_GF_Avec_x,
                                   AXB_GF_Avec_y, AXB_GF_Avec_z, AXB_GF_Psi};
const int kEvolvedRhsIds[NEVOLVED] = {
    AXB_GF_densrhs, AXB_GF_momxrhs, AXB_GF_momyrhs, AXB_GF_momzrhs,
    AXB_GF_taurhs,  AXB_GF_DYe_rhs, AXB_GF_DEntrhs, AXB_GF_Avec_x_rhs,
    AXB_GF_Avec_y_rhs, AXB_GF_Avec_z_rhs, AXB_GF_Psi_rhs};

// ---------------------------------------------------------------------------
// boundary fill, one direction per launch
// ---------------------------------------------------------------------------
struct BoundaryArgs {
  BoxDev b;
  double *f[AXB_NUM_GF];
  int cent[AXB_NUM_GF][3];
  int dir, bc_lo, bc_hi;
};

AXB_D int wrap_periodic(int i, int ng, int n) {
  int r = (i - ng) % n;
  if (r < 0)
    r += n;
  return ng + r;
}

// One thread per ghost point along `dir` (ng layers below, ng above), over
// the full extent of the other two directions of the field's centring
// (their ghosts included, so corners take the boundary rule of each
// direction in turn).  The boundary point is the outermost interior point
// of the centring along `dir`, the next one is its inner neighbour.
__global__ void __launch_bounds__(128) k_fill_dir(const BoundaryArgs a) {
  const int v = blockIdx.y;
  const BoxDev &b = a.b;
  const int d = a.dir, d1 = (d + 1) % 3, d2 = (d + 2) % 3;
  const int *c = a.cent[v];
  const int ng = b.ng;
  int N[3];
  for (int e = 0; e < 3; ++e)
    N[e] = b.n[e] + 2 * ng + (c[e] ? 0 : 1);
  const long long per_side = (long long)ng * N[d1] * N[d2];
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= 2 * per_side)
    return;
  const int side = g >= per_side;
  long long r = g - side * per_side;
  const int q = int(r % ng);
  r /= ng;
  const int t1 = int(r % N[d1]);
  const int t2 = int(r / N[d1]);
  const int lo_b = ng, hi_b = ng + b.n[d] - (c[d] ? 1 : 0);
  int gi, bi, ii;
  if (!side) {
    gi = q;
    bi = lo_b;
    ii = lo_b + 1;
  } else {
    gi = hi_b + 1 + q;
    bi = hi_b;
    ii = hi_b - 1;
  }
  int ijk[3];
  ijk[d1] = t1;
  ijk[d2] = t2;
  ijk[d] = gi;
  const long long G = b.at(ijk[0], ijk[1], ijk[2]);
  const long long sd = b.stride(d);
  const long long B = G + (long long)(bi - gi) * sd;
  double *f = a.f[v];
  const int type = side ? a.bc_hi : a.bc_lo;
  if (type == AXB_BC_PERIODIC) {
    const int n_per = b.n[d];
    const int src = wrap_periodic(gi, ng, n_per);
    f[G] = f[G + (long long)(src - gi) * sd];
  } else if (type == AXB_BC_NEUMANN) {
    f[G] = f[B];
  } else { // linear extrapolation from the two outermost interior points
    const long long Iin = G + (long long)(ii - gi) * sd;
    const double k = double(abs(gi - bi));
    f[G] = f[B] + k * (f[B] - f[Iin]);
  }
}

// ---------------------------------------------------------------------------
// general stage combination
// ---------------------------------------------------------------------------
constexpr int MAXSTATES = 4;
struct LincombArgs {
  BoxDev b;
  double *out[NEVOLVED];
  const double *s[MAXSTATES][NEVOLVED];
  const double *rhs[NEVOLVED];
  double coef[MAXSTATES], gdt;
  int nstates;
  int cent[NEVOLVED][3];
};

__global__ void __launch_bounds__(128) k_lincomb(const LincombArgs a) {
  const BoxDev &b = a.b;
  int i, j;
  const int k = b.ng + blockIdx.z;
  if (!b.row_ij(b.ng, b.n[0] + 1, b.ng, b.n[1] + 1, blockIdx, i, j))
    return;
  const long long I = b.at(i, j, k);
  const int ijk[3] = {i, j, k};
  for (int v = 0; v < NEVOLVED; ++v) {
    bool in = true;
    for (int d = 0; d < 3; ++d)
      in &= ijk[d] < b.ng + b.n[d] + (a.cent[v][d] ? 0 : 1);
    if (!in)
      continue;
    // states in order, then the RHS, each as one fused multiply-add
    double acc = a.coef[0] * a.s[0][v][I];
    for (int q = 1; q < a.nstates; ++q)
      acc = fma(a.coef[q], a.s[q][v][I], acc);
    a.out[v][I] = fma(a.gdt, a.rhs[v][I], acc);
  }
}

// ---------------------------------------------------------------------------
// grid functions between the caller's per-field layouts and the engine's
// ---------------------------------------------------------------------------
struct CopyArgs {
  BoxDev b;
  double *dst[AXB_NUM_GF];
  const double *src[AXB_NUM_GF];
  long long ssy[AXB_NUM_GF], ssz[AXB_NUM_GF]; // strides of the strided side
  int cent[AXB_NUM_GF][3];
  int to_engine; // 1: strided -> engine layout, 0: engine -> strided
};

// One thread per point of the field's centring extent (ghosts included).
__global__ void __launch_bounds__(128) k_copy_layout(const CopyArgs a) {
  const int v = blockIdx.y;
  const BoxDev &b = a.b;
  const int *c = a.cent[v];
  const int N0 = b.n[0] + 2 * b.ng + (c[0] ? 0 : 1);
  const int N1 = b.n[1] + 2 * b.ng + (c[1] ? 0 : 1);
  const int N2 = b.n[2] + 2 * b.ng + (c[2] ? 0 : 1);
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)N0 * N1 * N2)
    return;
  const int i = int(g % N0);
  const int j = int((g / N0) % N1);
  const int k = int(g / ((long long)N0 * N1));
  const long long E = b.at(i, j, k);
  const long long S = (long long)i + a.ssy[v] * j + a.ssz[v] * k;
  if (a.to_engine)
    a.dst[v][E] = a.src[v][S];
  else
    a.dst[v][S] = a.src[v][E];
}

int copy_layout(axb_ctx *c, const axb_box *box, const axb_fields *eng,
                const axb_fields_strided *str, const int *ids, int nids, int to_engine,
                cudaStream_t s) {
  if (!c || !box || !eng || !str || !ids || nids < 1 || nids > AXB_NUM_GF || box->ng < 0)
    return AXB_ERR_ARG;
  for (int d = 0; d < 3; ++d)
    if (box->n[d] < 1)
      return AXB_ERR_ARG;
  CopyArgs a;
  a.b = make_box(*box);
  a.to_engine = to_engine;
  long long gmax = 0;
  for (int q = 0; q < nids; ++q) {
    const int id = ids[q];
    if (id < 0 || id >= AXB_NUM_GF || !eng->gf[id] || !str->gf[id])
      return AXB_ERR_ARG;
    gf_centring(id, a.cent[q]);
    const long long N0 = box->n[0] + 2LL * box->ng + (a.cent[q][0] ? 0 : 1);
    const long long N1 = box->n[1] + 2LL * box->ng + (a.cent[q][1] ? 0 : 1);
    const long long N2 = box->n[2] + 2LL * box->ng + (a.cent[q][2] ? 0 : 1);
    // the strided side must hold its centring's points without overlap
    if (str->sy[id] < N0 || str->sz[id] < str->sy[id] * N1)
      return AXB_ERR_ARG;
    a.ssy[q] = str->sy[id];
    a.ssz[q] = str->sz[id];
    if (to_engine) {
      a.src[q] = str->gf[id];
      a.dst[q] = eng->gf[id];
    } else {
      a.src[q] = eng->gf[id];
      a.dst[q] = str->gf[id];
    }
    gmax = std::max(gmax, N0 * N1 * N2);
  }
  const dim3 grid(unsigned((gmax + 127) / 128), nids);
  k_copy_layout<<<grid, 128, 0, s>>>(a);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

bool bc_valid(int t) {
  return t == AXB_BC_PERIODIC || t == AXB_BC_NEUMANN || t == AXB_BC_LINEAR;
}

} // namespace

// Outer-boundary fill of the grid functions `ids[0..nids)`, each with its
// own centring: the ghost layers of every face take the face's rule
// (bc[0..5] = x-lower, x-upper, y-lower, y-upper, z-lower, z-upper), one
// direction after the other.
AXB_API int axb_fill_boundary(axb_ctx *c, const axb_box *box, const axb_fields *f,
                              const int *ids, int nids, const int bc[6], void *stream) {
  if (!c || !box || !f || !ids || !bc || nids < 1 || nids > AXB_NUM_GF)
    return AXB_ERR_ARG;
  if (box->ng < 1)
    return AXB_ERR_GHOSTS;
  for (int q = 0; q < 6; ++q)
    if (!bc_valid(bc[q]))
      return AXB_ERR_ARG;
  for (int d = 0; d < 3; ++d) {
    if (box->n[d] < 2)
      return AXB_ERR_ARG; // linear extrapolation needs two interior points
    if ((bc[2 * d] == AXB_BC_PERIODIC) != (bc[2 * d + 1] == AXB_BC_PERIODIC))
      return AXB_ERR_ARG; // periodic on both faces of an axis or on neither
    if (bc[2 * d] == AXB_BC_PERIODIC && box->n[d] < box->ng)
      return AXB_ERR_ARG;
  }
  BoundaryArgs a;
  a.b = make_box(*box);
  long long gmax = 0;
  for (int q = 0; q < nids; ++q) {
    if (ids[q] < 0 || ids[q] >= AXB_NUM_GF || !f->gf[ids[q]])
      return AXB_ERR_ARG;
    a.f[q] = f->gf[ids[q]];
    gf_centring(ids[q], a.cent[q]);
  }
  cudaStream_t s = (cudaStream_t)stream;
  axb_mark(c, AXB_R_SYNC, s, true);
  for (int d = 0; d < 3; ++d) {
    a.dir = d;
    a.bc_lo = bc[2 * d];
    a.bc_hi = bc[2 * d + 1];
    gmax = 0;
    const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
    for (int q = 0; q < nids; ++q) {
      const long long n1 = box->n[d1] + 2 * box->ng + (a.cent[q][d1] ? 0 : 1);
      const long long n2 = box->n[d2] + 2 * box->ng + (a.cent[q][d2] ? 0 : 1);
      gmax = std::max(gmax, 2LL * box->ng * n1 * n2);
    }
    const dim3 grid(unsigned((gmax + 127) / 128), nids);
    k_fill_dir<<<grid, 128, 0, s>>>(a);
  }
  axb_mark(c, AXB_R_SYNC, s, false);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

// out = sum_q coef[q] * states[q] + gdt * RHS on the interiors of the 11
// evolved variables.  `out` may be one of the states.
AXB_API int axb_rk_lincomb(axb_ctx *c, const axb_box *box, const axb_fields *out,
                           int nstates, const double *coef, const axb_fields *const *states,
                           double gdt, const axb_fields *rhs, void *stream) {
  if (!c || !box || !out || !coef || !states || !rhs || nstates < 1 ||
      nstates > MAXSTATES)
    return AXB_ERR_ARG;
  LincombArgs a;
  a.b = make_box(*box);
  a.nstates = nstates;
  a.gdt = gdt;
  for (int q = 0; q < nstates; ++q) {
    if (!states[q])
      return AXB_ERR_ARG;
    a.coef[q] = coef[q];
  }
  for (int v = 0; v < NEVOLVED; ++v) {
    a.out[v] = out->gf[kEvolvedIds[v]];
    a.rhs[v] = rhs->gf[kEvolvedRhsIds[v]];
    if (!a.out[v] || !a.rhs[v])
      return AXB_ERR_ARG;
    for (int q = 0; q < nstates; ++q) {
      a.s[q][v] = states[q]->gf[kEvolvedIds[v]];
      if (!a.s[q][v])
        return AXB_ERR_ARG;
    }
    gf_centring(kEvolvedIds[v], a.cent[v]);
  }
  const int T = 128;
  const dim3 grid((box->n[0] + 1 + T - 1) / T, box->n[1] + 1, box->n[2] + 1);
  cudaStream_t s = (cudaStream_t)stream;
  axb_mark(c, AXB_R_STAGE, s, true);
  k_lincomb<<<grid, T, 0, s>>>(a);
  axb_mark(c, AXB_R_STAGE, s, false);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

// Grid functions whose centrings have their own extents and strides (as
// CarpetX allocates them) into the engine's one-layout box, and back.
AXB_API int axb_import_fields(axb_ctx *c, const axb_box *box, const axb_fields_strided *src,
                              const int *ids, int nids, const axb_fields *dst, void *stream) {
  return copy_layout(c, box, dst, src, ids, nids, 1, (cudaStream_t)stream);
}
AXB_API int axb_export_fields(axb_ctx *c, const axb_box *box, const axb_fields *src,
                              const int *ids, int nids, const axb_fields_strided *dst,
                              void *stream) {
  return copy_layout(c, box, src, dst, ids, nids, 0, (cudaStream_t)stream);
}
