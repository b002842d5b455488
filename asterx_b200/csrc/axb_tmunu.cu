// The fluid's stress-energy tensor on the vertices and the regrid error
// estimate: the two scheduled routines of AsterX outside the RHS and
// post-step groups that read the evolved state every step.
//
//   k_tmunu<ORDER, ZVEC>   AsterX_Tmunu (AsterX/src/tmunu.cxx:19-178): the
//                          cell-centred primitives interpolated to each
//                          interior vertex (AsterUtils/src/aster_interp.hxx:
//                          97-148, order 2 or 4), T_{mu nu} of the ideal
//                          MHD fluid added to eTtt .. eTzz
//   k_regrid_error<M>      AsterX_EstimateError (AsterX/src/
//                          estimate_error.cxx:70-144) with the indicators of
//                          AsterX/src/estimate_error.hxx:14-86
//
// Both are HBM-bound point loops (one thread per point, rows of 128 along
// x, neighbours from L1/L2).  This file is compiled without multiply-add
// contraction and keeps the reference's operation order (sums from left to
// right, products left-associated as written), so the results are the
// reference's bits: IEEE division and square root round the same on both.
#include <algorithm>

#include "axb_internal.hxx"

using namespace axb;

namespace {

// ---------------------------------------------------------------------------
// AsterX_Tmunu
// ---------------------------------------------------------------------------
struct TmunuArgs {
  BoxDev b;
  const double *rho, *eps, *press, *v[3], *B[3];
  const double *g[6], *alp, *beta[3];
  double *eT[10];
};

// Order 2: the 8 cells around vertex I (cell I - di - dj - dk), summed in
// the reference's loop order (dk, dj, di), divided by 8.
AXB_D double c2v2(const double *__restrict__ f, long long I, long long sy, long long sz) {
  double s = 0.0;
#pragma unroll
  for (int dk = 0; dk < 2; ++dk)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj)
#pragma unroll
      for (int di = 0; di < 2; ++di)
        s += __ldg(f + I - di - dj * sy - dk * sz);
  return s / 8.0;
}

// Order 4: the cubic Lagrange weights (-1, 9, 9, -1)/16 on cells I-2 .. I+1
// along each direction, applied direction i first, then j, then k, for the
// three cyclic orders (i, j, k) = (x, y, z), (y, z, x), (z, x, y), all
// twelve final terms accumulated in one running sum, divided by 3.
AXB_D double c2v4(const double *__restrict__ f, long long I, const long long st[3]) {
  const double wt[4] = {-1.0 / 16.0, 9.0 / 16.0, 9.0 / 16.0, -1.0 / 16.0};
  double avg = 0.0;
#pragma unroll 1
  for (int i = 0; i < 3; ++i) {
    const int j = (i == 0) ? 1 : ((i == 1) ? 2 : 0);
    const int k = (i == 0) ? 2 : ((i == 1) ? 0 : 1);
    double gj[4];
#pragma unroll
    for (int dk = 0; dk < 4; ++dk) {
      double gi[4];
#pragma unroll
      for (int dj = 0; dj < 4; ++dj) {
        double s = 0.0;
        const long long base = I + st[j] * (dj - 2) + st[k] * (dk - 2);
#pragma unroll
        for (int di = 0; di < 4; ++di)
          s += wt[di] * __ldg(f + base + st[i] * (di - 2));
        gi[dj] = s;
      }
      double s = 0.0;
#pragma unroll
      for (int dj = 0; dj < 4; ++dj)
        s += wt[dj] * gi[dj];
      gj[dk] = s;
    }
#pragma unroll
    for (int dk = 0; dk < 4; ++dk)
      avg += wt[dk] * gj[dk];
  }
  return avg / 3.0;
}

template <int ORDER>
AXB_D double c2v(const double *__restrict__ f, long long I, const long long st[3]) {
  if constexpr (ORDER == 2)
    return c2v2(f, I, st[1], st[2]);
  else
    return c2v4(f, I, st);
}

// Interior vertices [ng, ng + n] per axis; x along the block's threads.
template <int ORDER, bool ZVEC>
__global__ void __launch_bounds__(128) k_tmunu(const TmunuArgs a) {
  const BoxDev &b = a.b;
  const int i = b.ng + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = b.ng + blockIdx.y;
  const int k = b.ng + blockIdx.z;
  if (i > b.ng + b.n[0])
    return;
  const long long I = b.at(i, j, k);
  const long long st[3] = {1, b.sy, b.sz};

  const double rho_avg = c2v<ORDER>(a.rho, I, st);
  const double eps_avg = c2v<ORDER>(a.eps, I, st);
  const double press_avg = c2v<ORDER>(a.press, I, st);
  double Bup[3];
  for (int d = 0; d < 3; ++d)
    Bup[d] = c2v<ORDER>(a.B[d], I, st);

  const sym3 g{__ldg(a.g[0] + I), __ldg(a.g[1] + I), __ldg(a.g[2] + I),
               __ldg(a.g[3] + I), __ldg(a.g[4] + I), __ldg(a.g[5] + I)};
  const double alp = __ldg(a.alp + I);
  const double beta_up[3] = {__ldg(a.beta[0] + I), __ldg(a.beta[1] + I),
                             __ldg(a.beta[2] + I)};
  double beta_low[3];
  lower3(g, beta_up, beta_low);
  const double beta_sq = dot3(beta_low, beta_up);

  double vup[3], vlow[3], w;
  if constexpr (!ZVEC) {
    for (int d = 0; d < 3; ++d)
      vup[d] = c2v<ORDER>(a.v[d], I, st);
    lower3(g, vup, vlow);
    w = 1.0 / sqrt(1.0 - dot3(vup, vlow));
  } else {
    double zup[3], zlow[3];
    for (int d = 0; d < 3; ++d)
      zup[d] = c2v<ORDER>(a.v[d], I, st);
    lower3(g, zup, zlow);
    w = sqrt(1.0 + dot3(zup, zlow));
    for (int d = 0; d < 3; ++d) {
      vup[d] = zup[d] / w;
      vlow[d] = zlow[d] / w;
    }
  }

  const double rhW2 = (rho_avg * (1.0 + eps_avg) + press_avg) * w * w;
  const double ut_low = -alp + dot3(beta_low, vup);
  double ui_up[3];
  for (int d = 0; d < 3; ++d)
    ui_up[d] = vup[d] - beta_up[d] / alp;
  const double bst_up = w * (dot3(Bup, vlow)) / alp;
  double bsi_up[3];
  for (int d = 0; d < 3; ++d)
    bsi_up[d] = (Bup[d] + alp * bst_up * w * ui_up[d]) / w;
  const double gtt = -alp * alp + beta_sq;
  const double bst_low = bst_up * gtt + dot3(bsi_up, beta_low);
  double gb[3], bsi_low[3];
  lower3(g, bsi_up, gb);
  for (int d = 0; d < 3; ++d)
    bsi_low[d] = bst_up * beta_low[d] + gb[d];
  const double bs2 = bst_up * bst_low + dot3(bsi_up, bsi_low);
  const double w2 = w * w;

  const double t00 = rhW2 * ut_low * ut_low + press_avg * gtt +
                     (w2 * ut_low * ut_low + 0.5 * gtt) * bs2 - bst_low * bst_low;
  double t0[3];
  for (int d = 0; d < 3; ++d)
    t0[d] = rhW2 * ut_low * vlow[d] + press_avg * beta_low[d] +
            (w2 * ut_low * vlow[d] + 0.5 * beta_low[d]) * bs2 - bst_low * bsi_low[d];
  auto tij = [&](int p, int q) {
    return rhW2 * vlow[p] * vlow[q] + press_avg * g(p, q) +
           (w2 * vlow[p] * vlow[q] + 0.5 * g(p, q)) * bs2 - bsi_low[p] * bsi_low[q];
  };
  const double t[10] = {t00,       t0[0],     t0[1],     t0[2],     tij(0, 0),
                        tij(0, 1), tij(0, 2), tij(1, 1), tij(1, 2), tij(2, 2)};
#pragma unroll
  for (int c = 0; c < 10; ++c)
    a.eT[c][I] = a.eT[c][I] + t[c];
}

template <int ORDER, bool ZVEC>
void launch_tmunu(const TmunuArgs &a, cudaStream_t s) {
  const dim3 grid((a.b.n[0] + 1 + 127) / 128, a.b.n[1] + 1, a.b.n[2] + 1);
  k_tmunu<ORDER, ZVEC><<<grid, 128, 0, s>>>(a);
}

// ---------------------------------------------------------------------------
// AsterX_EstimateError
// ---------------------------------------------------------------------------
constexpr int MAXVARS = 9; // the reference asserts NregridVars < 10

struct ErrorArgs {
  BoxDev b;
  const double *var[MAXVARS];
  int nvars;
  double epsilon_err;
  double *err;
};

// std::max over an initializer list: the first largest, NaN kept only when
// it comes first
AXB_D double max_il(double a, double b) { return (a < b) ? b : a; }

template <int M>
AXB_D double indicator(const double *__restrict__ f, long long I, const long long st[3],
                       double epsilon_err) {
  if constexpr (M == AXB_REGRID_FIRST_GRAD) {
    double errp = 0.0, errm = 0.0;
    const double v0 = __ldg(f + I);
    for (int d = 0; d < 3; ++d) {
      const double vm = __ldg(f + I - st[d]), vp = __ldg(f + I + st[d]);
      errp += (vp - v0) * (vp - v0);
      errm += (v0 - vm) * (v0 - vm);
    }
    return sqrt(max_il(errp, errm));
  } else {
    double err = 0.0;
    const double v0 = __ldg(f + I);
    for (int d = 0; d < 3; ++d) {
      const double vm = __ldg(f + I - st[d]), vp = __ldg(f + I + st[d]);
      if constexpr (M == AXB_REGRID_FIRST_DERIV) {
        err = max_il(max_il(err, fabs(v0 - vm)), fabs(vp - v0));
      } else if constexpr (M == AXB_REGRID_SECOND_DERIV) {
        err = max_il(err, fabs(vp + vm - 2 * v0));
      } else {
        const double dp = vp - v0, dm = v0 - vm;
        const double varsigma = fabs(vp) + 2 * fabs(v0) + fabs(vm);
        const double num = fabs(dp - dm) * fabs(dp - dm);
        const double den = (fabs(dp) + fabs(dm) + epsilon_err * varsigma) *
                           (fabs(dp) + fabs(dm) + epsilon_err * varsigma);
        err = max_il(err, sqrt(num / den));
      }
    }
    return err;
  }
}

// Interior cells; x along the block's threads.
template <int M> __global__ void __launch_bounds__(128) k_regrid_error(const ErrorArgs a) {
  const BoxDev &b = a.b;
  const int i = b.ng + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = b.ng + blockIdx.y;
  const int k = b.ng + blockIdx.z;
  if (i >= b.ng + b.n[0])
    return;
  const long long I = b.at(i, j, k);
  const long long st[3] = {1, b.sy, b.sz};
  double e = 0.0;
  for (int v = 0; v < a.nvars; ++v)
    e = max_il(e, indicator<M>(a.var[v], I, st, a.epsilon_err));
  a.err[I] = e;
}

template <int M> void launch_error(const ErrorArgs &a, cudaStream_t s) {
  const dim3 grid((a.b.n[0] + 127) / 128, a.b.n[1], a.b.n[2]);
  k_regrid_error<M><<<grid, 128, 0, s>>>(a);
}

bool grid_ok(const axb_box &b, int extra) {
  for (int d = 0; d < 3; ++d)
    if (b.n[d] < 1 || b.n[d] + extra > 65535)
      return false;
  return true;
}

} // namespace

AXB_API int axb_tmunu(axb_ctx *c, const axb_box *box, const axb_fields *f,
                      const axb_params *p, int interp_order, double *const eT[10],
                      void *stream) {
  if (!c || !box || !f || !p || !eT)
    return AXB_ERR_ARG;
  if (interp_order != 2 && interp_order != 4)
    return AXB_ERR_ARG;
  if (box->ng < (interp_order == 4 ? 2 : 1))
    return AXB_ERR_GHOSTS;
  if (!grid_ok(*box, 1))
    return AXB_ERR_ARG;
  if (p->recon_type != AXB_RECVAR_V && p->recon_type != AXB_RECVAR_Z &&
      p->recon_type != AXB_RECVAR_S)
    return AXB_ERR_ARG;
  TmunuArgs a;
  a.b = make_box(*box);
  // s_vec reconstructs svec at the faces; the vertex tensor interpolates
  // the velocity as v_vec does (tmunu.cxx:35 tests recon_type == "v_vec"
  // only, so s_vec takes the zvec branch there): the zvec grid functions
  // are read for both z_vec and s_vec
  const bool zv = p->recon_type != AXB_RECVAR_V;
  const double *req[] = {f->gf[AXB_GF_rho], f->gf[AXB_GF_eps], f->gf[AXB_GF_press],
                         f->gf[AXB_GF_alp]};
  for (const double *q : req)
    if (!q)
      return AXB_ERR_ARG;
  a.rho = f->gf[AXB_GF_rho];
  a.eps = f->gf[AXB_GF_eps];
  a.press = f->gf[AXB_GF_press];
  a.alp = f->gf[AXB_GF_alp];
  for (int d = 0; d < 3; ++d) {
    a.v[d] = f->gf[(zv ? AXB_GF_zvec_x : AXB_GF_velx) + d];
    a.B[d] = f->gf[AXB_GF_Bvecx + d];
    a.beta[d] = f->gf[AXB_GF_betax + d];
    if (!a.v[d] || !a.B[d] || !a.beta[d])
      return AXB_ERR_ARG;
  }
  for (int q = 0; q < 6; ++q) {
    a.g[q] = f->gf[AXB_GF_gxx + q];
    if (!a.g[q])
      return AXB_ERR_ARG;
  }
  for (int q = 0; q < 10; ++q) {
    a.eT[q] = eT[q];
    if (!eT[q])
      return AXB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  axb_mark(c, AXB_R_TMUNU, s, true);
  if (interp_order == 2)
    zv ? launch_tmunu<2, true>(a, s) : launch_tmunu<2, false>(a, s);
  else
    zv ? launch_tmunu<4, true>(a, s) : launch_tmunu<4, false>(a, s);
  axb_mark(c, AXB_R_TMUNU, s, false);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

AXB_API int axb_estimate_error(axb_ctx *c, const axb_box *box, const double *const *vars,
                               int nvars, int method, double epsilon_err,
                               double *regrid_error, void *stream) {
  if (!c || !box || !vars || !regrid_error || nvars < 1 || nvars > MAXVARS)
    return AXB_ERR_ARG;
  if (method < AXB_REGRID_FIRST_DERIV || method > AXB_REGRID_FIRST_GRAD)
    return AXB_ERR_ARG;
  if (box->ng < 1)
    return AXB_ERR_GHOSTS;
  if (!grid_ok(*box, 0))
    return AXB_ERR_ARG;
  ErrorArgs a;
  a.b = make_box(*box);
  a.nvars = nvars;
  a.epsilon_err = epsilon_err;
  a.err = regrid_error;
  for (int v = 0; v < nvars; ++v) {
    if (!vars[v])
      return AXB_ERR_ARG;
    a.var[v] = vars[v];
  }
  cudaStream_t s = (cudaStream_t)stream;
  axb_mark(c, AXB_R_ERROR, s, true);
  switch (method) {
  case AXB_REGRID_FIRST_DERIV:
    launch_error<AXB_REGRID_FIRST_DERIV>(a, s);
    break;
  case AXB_REGRID_SECOND_DERIV:
    launch_error<AXB_REGRID_SECOND_DERIV>(a, s);
    break;
  case AXB_REGRID_SECOND_DERIV_NORM:
    launch_error<AXB_REGRID_SECOND_DERIV_NORM>(a, s);
    break;
  default:
    launch_error<AXB_REGRID_FIRST_GRAD>(a, s);
    break;
  }
  axb_mark(c, AXB_R_ERROR, s, false);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}
