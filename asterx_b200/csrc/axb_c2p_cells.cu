// Independent-cell recovery with the optional learned initial guess.
#include "axb_c2p_box.cuh"
#include "axb_mlp.cuh"

using namespace axb;

// ---------------------------------------------------------------------------
// Independent-cell recovery (the per-cell body of AsterX_Con2Prim_typeEoS,
// con2prim.cxx:137-416, without grid, mask or graded atmosphere), with the
// optional learned initial guess.
// ---------------------------------------------------------------------------
namespace axb {
MlpDev mlp_device_view(const axb_mlp *m);
int mlp_nf(const axb_mlp *m);
int launch_mlp_guess(const axb_cells &c, const axb_mlp *m, float2 *guess, DevStatus *status,
                     cudaStream_t s);

struct C2PCellsArgs {
  axb_cells c;
  C2PParams cp;
  int c2p_prime, c2p_second, use_entropy_fix;
  Atmo atmo;
  double gamma_noble, Zmin;
  int use_mlp;
  double bracket;
  MlpDev mlp;
  DevStatus *status;
};

template <class EOS>
AXB_D void run_solver_cells(int which, const EOS &eos, const C2PCellsArgs &a, Prim &pv,
                            Prim &seeds, Cons &cv, const sym3 &glo, Report &rep,
                            double zguess, double vsqguess, double xlo, double xhi) {
  if (which == AXB_C2P_NOBLE)
    noble_solve(eos, a.cp, a.atmo, a.gamma_noble, a.Zmin, pv, seeds, cv, glo, rep, zguess,
                vsqguess);
  else if (which == AXB_C2P_PALENZUELA)
    palenzuela_solve(eos, a.cp, a.atmo, pv, cv, glo, rep, xlo, xhi);
  else if (which == AXB_C2P_ENTROPY)
    entropy_solve(eos, a.cp, a.atmo, pv, cv, glo, rep);
}

template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_MINB)
    k_c2p_cells(const C2PCellsArgs a, const EOS eos) {
  __shared__ unsigned int s_hist[64];
  for (int q = threadIdx.x; q < 64; q += blockDim.x)
    s_hist[q] = 0;
  __syncthreads();
  const axb_cells &c = a.c;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < c.n;
  Cons cv;
  sym3 glo{1, 0, 0, 1, 0, 1};
  if (valid) {
    cv.dens = c.dens[i];
    for (int q = 0; q < 3; ++q) {
      cv.mom[q] = c.mom[q][i];
      cv.dBvec[q] = c.dB[q][i];
    }
    cv.tau = c.tau[i];
    cv.DYe = c.DYe[i];
    cv.DEnt = c.DEnt ? c.DEnt[i] : 0.0;
    glo = sym3{c.g[0][i], c.g[1][i], c.g[2][i], c.g[3][i], c.g[4][i], c.g[5][i]};
  }
  // learned guess (x = h W, W) from k_mlp_guess_tc
  double zguess = -1.0, vsqguess = -1.0, xlo = -1.0, xhi = -1.0;
  if (a.use_mlp && valid) {
    const float2 gs = reinterpret_cast<const float2 *>(c.guess)[i];
    const double x = gs.x, W = gs.y;
    zguess = cv.dens / sqrt(det3(glo)) * x; // Z = rho h W^2 = D (h W)
    vsqguess = 1.0 - 1.0 / (W * W);
    xlo = x * (1.0 - a.bracket);
    xhi = x * (1.0 + a.bracket);
    if (!(zguess > 0.0 && zguess < 1e300 && vsqguess >= 0.0 && vsqguess < 1.0))
      zguess = vsqguess = xlo = xhi = -1.0;
  }
  int iters_first = -1;
  bool failed = false, fallback = false;
  if (valid) {
    const double sqrt_detg = sqrt(det3(glo));
    const double isg = 1.0 / sqrt_detg;
    const double Bup[3] = {cv.dBvec[0] * isg, cv.dBvec[1] * isg, cv.dBvec[2] * isg};
    Prim pv;
    pv.set_nan();
    Prim seeds;
    if (c.seed_rho) {
      seeds.rho = c.seed_rho[i];
      seeds.eps = c.seed_eps[i];
      seeds.Ye = c.seed_Ye[i];
      for (int q = 0; q < 3; ++q)
        seeds.vel[q] = c.seed_vel[q][i];
      seeds.temperature = c.seed_temperature ? c.seed_temperature[i] : a.atmo.temp;
    } else { // cold start
      seeds.rho = cv.dens / sqrt_detg;
      seeds.eps = a.atmo.eps;
      seeds.Ye = cv.DYe / cv.dens;
      for (int q = 0; q < 3; ++q)
        seeds.vel[q] = 0.0;
      seeds.temperature = a.atmo.temp;
    }
    // the seed velocity is limited as in con2prim.cxx:168-209
    double v_low[3];
    lower3(glo, seeds.vel, v_low);
    const double vsq = dot3(v_low, seeds.vel);
    double zsq;
    if (vsq >= 1.0) {
      const double wlim = sqrt(1.0 + a.cp.vw_lim * a.cp.vw_lim);
      const double vlim = a.cp.vw_lim / wlim;
      for (int q = 0; q < 3; ++q)
        seeds.vel[q] *= vlim / sqrt(vsq);
      zsq = a.cp.vw_lim * a.cp.vw_lim;
    } else {
      zsq = vsq / (1.0 - vsq);
    }
    {
      double e = seeds.eps;
      seeds.press = eos.press_from_valid_rho_eps_ye(seeds.rho, e, seeds.Ye);
    }
    seeds.entropy = 0.0;
    for (int q = 0; q < 3; ++q) {
      seeds.Bvec[q] = Bup[q];
      seeds.E[q] = 0.0;
    }
    seeds.w_lor = sqrt(1.0 + zsq);
    int code;
    if (cv.dens <= sqrt_detg * a.atmo.rho_cut) {
      for (int q = 0; q < 3; ++q)
        pv.Bvec[q] = Bup[q];
      a.atmo.set(pv, cv, glo);
      code = AXB_C2P_ATMO;
      cons_floors(cv, glo);
    } else {
      cons_floors(cv, glo);
      Report r1, r2;
      code = AXB_C2P_PRIME;
      const bool guessed = zguess >= 0.0;
      const Prim seeds_plain = seeds; // the first scheme may overwrite its seeds
      run_solver_cells(a.c2p_prime, eos, a, pv, seeds, cv, glo, r1, zguess, vsqguess, xlo,
                       xhi);
      iters_first = r1.iters;
      if (r1.failed() && guessed) {
        // the guess led the first scheme astray: the plain cold start
        // (c2p_2DNoble.hxx:374-393, the plain bracket), then the plain cascade
        fallback = true;
        seeds = seeds_plain;
        pv.set_nan();
        Report rr;
        run_solver_cells(a.c2p_prime, eos, a, pv, seeds, cv, glo, rr, -1.0, -1.0, -1.0, -1.0);
        iters_first += rr.iters;
        r1 = rr;
      }
      if (r1.failed()) {
        code = AXB_C2P_SECOND;
        run_solver_cells(a.c2p_second, eos, a, pv, seeds, cv, glo, r2, -1.0, -1.0, -1.0,
                         -1.0);
      }
      bool recovered = false;
      if (r1.failed() && r2.failed() && a.use_entropy_fix) {
        Report re;
        entropy_solve(eos, a.cp, a.atmo, pv, cv, glo, re);
        recovered = !re.failed();
        if (recovered)
          code = AXB_C2P_ENTROPY_OK;
      }
      if (r1.failed() && r2.failed() && !recovered) {
        code = AXB_C2P_FAIL;
        failed = true;
        for (int q = 0; q < 3; ++q) {
          cv.dBvec[q] = sqrt_detg * Bup[q];
          pv.Bvec[q] = Bup[q];
        }
        a.atmo.set(pv, cv, glo);
      }
    }
    if (c.flag)
      c.flag[i] = code;
    if (c.fallback)
      c.fallback[i] = fallback ? 1.0 : 0.0;
    if (c.iters)
      c.iters[i] = iters_first;
    if (c.rho)
      c.rho[i] = pv.rho;
    if (c.eps)
      c.eps[i] = pv.eps;
    if (c.press)
      c.press[i] = pv.press;
    for (int q = 0; q < 3; ++q)
      if (c.vel[q])
        c.vel[q][i] = pv.vel[q];
    if (c.w_lorentz)
      c.w_lorentz[i] = pv.w_lor;
    if (c.Ye)
      c.Ye[i] = pv.Ye;
    if (c.temperature)
      c.temperature[i] = pv.temperature;
    if (c.entropy)
      c.entropy[i] = pv.entropy;
  }
  const unsigned nfail = __popc(__ballot_sync(0xffffffffu, failed));
  if (nfail && (threadIdx.x % 32) == 0) {
    atomicAdd(&a.status->c2p_fail_count, nfail);
    atomicOr(&a.status->error_word, AXB_EW_C2P_FAIL);
  }
  if (iters_first >= 0)
    atomicAdd(&s_hist[min(iters_first, 63)], 1u);
  __syncthreads();
  for (int q = threadIdx.x; q < 64; q += blockDim.x)
    if (s_hist[q])
      atomicAdd(&a.status->c2p_iter_hist[q], (unsigned long long)s_hist[q]);
}
} // namespace axb

AXB_API int axb_c2p_cells(axb_ctx *ctx, const axb_cells *cells, const axb_params *p,
                          const axb_eos *eos, const axb_mlp *mlp, void *stream) {
  if (!ctx || !cells || !p || !eos || cells->n < 0)
    return AXB_ERR_ARG;
  if (!cells->dens || !cells->tau || !cells->DYe)
    return AXB_ERR_ARG;
  for (int q = 0; q < 3; ++q)
    if (!cells->mom[q] || !cells->dB[q])
      return AXB_ERR_ARG;
  for (int q = 0; q < 6; ++q)
    if (!cells->g[q])
      return AXB_ERR_ARG;
  if (cells->seed_rho && (!cells->seed_eps || !cells->seed_Ye || !cells->seed_vel[0] ||
                          !cells->seed_vel[1] || !cells->seed_vel[2]))
    return AXB_ERR_ARG;
  auto ok_solver = [](int s) {
    return s == AXB_C2P_NOBLE || s == AXB_C2P_PALENZUELA || s == AXB_C2P_ENTROPY;
  };
  if (!ok_solver(p->c2p_prime) || !(ok_solver(p->c2p_second) || p->c2p_second == AXB_C2P_NONE))
    return AXB_ERR_UNSUPPORTED;
  const bool entropy = p->use_entropy_fix || p->c2p_prime == AXB_C2P_ENTROPY ||
                       p->c2p_second == AXB_C2P_ENTROPY;
  if (entropy && eos->kind != 0)
    return AXB_ERR_UNSUPPORTED; // p(rho, kappa) is not defined for a table
  if (entropy && !cells->DEnt)
    return AXB_ERR_ARG; // the entropy scheme reads the conserved entropy
  if (!(p->c2p_tol > 0) || p->max_iter < 1)
    return AXB_ERR_ARG;
  C2PCellsArgs a;
  a.c = *cells;
  a.cp = make_c2p_params(*p);
  a.c2p_prime = p->c2p_prime;
  a.c2p_second = p->c2p_second;
  a.use_entropy_fix = p->use_entropy_fix;
  a.status = ctx->status;
  a.use_mlp = mlp != nullptr;
  a.bracket = 0.0;
  if (mlp) {
    if (!cells->guess)
      return AXB_ERR_ARG;
    a.mlp = mlp_device_view(mlp);
    a.bracket = a.mlp.bracket;
    if (eos->kind == 1 && mlp_nf(mlp) != 9)
      return AXB_ERR_ARG; // the tabulated guess takes Ye as a ninth input
  }
  // uniform atmosphere as for a box inside r_atmo (host_atmosphere)
  C2PBoxArgs hb{};
  hb.thermal_eos_atmo = p->thermal_eos_atmo;
  hb.use_press_atmo = p->use_press_atmo;
  hb.rho_abs_min = p->rho_abs_min;
  hb.p_atmo = p->p_atmo;
  hb.t_atmo = p->t_atmo;
  hb.Ye_atmo = p->Ye_atmo;
  hb.atmo_tol = p->atmo_tol;
  hb.poly = eos->poly;
  if (eos->kind == 0) {
    a.gamma_noble = eos->ideal.gamma;
    a.Zmin = eos->ideal.rgrho.min;
    a.atmo = host_atmosphere(hb, eos->ideal);
  } else if (eos->kind == 1) {
    if (p->thermal_eos_atmo && p->use_press_atmo)
      return AXB_ERR_UNSUPPORTED;
    a.gamma_noble = std::numeric_limits<double>::quiet_NaN();
    a.Zmin = eos->tab_h.rgrho.min;
    a.atmo = host_atmosphere(hb, eos->tab_h);
  } else {
    return AXB_ERR_UNSUPPORTED;
  }
  if (cells->n == 0)
    return AXB_OK;
  const long long blocks = (cells->n + 127) / 128;
  if (blocks > 0x7fffffffLL)
    return AXB_ERR_TOO_LARGE;
  cudaStream_t s = (cudaStream_t)stream;
  if (mlp) {
    axb_mark(ctx, AXB_R_MLP, s, true);
    const int rc = launch_mlp_guess(*cells, mlp, reinterpret_cast<float2 *>(cells->guess),
                                   ctx->status, s);
    axb_mark(ctx, AXB_R_MLP, s, false);
    if (rc)
      return rc;
  }
  axb_mark(ctx, AXB_R_C2P_CELLS, s, true);
  if (eos->kind == 1)
    k_c2p_cells<<<(unsigned)blocks, 128, 0, s>>>(a, tab_for_launch(*eos, a.status));
  else
    k_c2p_cells<<<(unsigned)blocks, 128, 0, s>>>(a, eos->ideal);
  axb_mark(ctx, AXB_R_C2P_CELLS, s, false);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

