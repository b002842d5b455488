// Con2PrimFactory primitive recovery on the device.
//
//   Noble 2D Newton-Raphson  Con2PrimFactory/src/c2p_2DNoble.hxx:192-594
//   Palenzuela 1D root        Con2PrimFactory/src/c2p_1DPalenzuela.hxx:142-556
//   floors and ceilings       Con2PrimFactory/src/c2p.hxx:86-216,330-369
//   BH-interior treatment     Con2PrimFactory/src/c2p.hxx:218-328
//   atmosphere                Con2PrimFactory/src/atmo.hxx:49-82
//   prim -> cons              Con2PrimFactory/src/cons.hxx:48-91
//
// The functions mirror the reference's control flow step by step, including
// its quirks (a non-finite Newton residual marks the report failed after
// convergence but the primitives are still written; Palenzuela takes the
// bracket midpoint), so that a cell follows the same branch as on the CPU.
#pragma once

#include "axb_common.cuh"
#include "axb_eos.cuh"

namespace axb {

struct Prim {
  double rho, eps, Ye, press, temperature, entropy;
  double vel[3];
  double w_lor;
  double Bvec[3];
  double E[3];
  AXB_HD void set_nan() {
    const double n = nan("");
    rho = eps = Ye = press = temperature = entropy = w_lor = n;
    for (int i = 0; i < 3; ++i)
      vel[i] = Bvec[i] = E[i] = n;
  }
};

struct Cons {
  double dens, mom[3], tau, DYe, DEnt, dBvec[3];
  AXB_HD void set_nan() {
    const double n = nan("");
    dens = tau = DYe = DEnt = n;
    for (int i = 0; i < 3; ++i)
      mom[i] = dBvec[i] = n;
  }
  AXB_HD void scale(double s) { // multiply every component (densitise)
    dens *= s;
    tau *= s;
    for (int i = 0; i < 3; ++i) {
      mom[i] *= s;
      dBvec[i] *= s;
    }
    DYe *= s;
    DEnt *= s;
  }
  AXB_HD void unscale(double s) { // divide every component (undensitise)
    // one division and eight products instead of eight divisions
    // (last-ulp differences)
    const double is = 1.0 / s;
    dens *= is;
    tau *= is;
    for (int i = 0; i < 3; ++i)
      mom[i] *= is;
    for (int i = 0; i < 3; ++i)
      dBvec[i] *= is;
    DYe *= is;
    DEnt *= is;
  }
};

// c2p_report (Con2PrimFactory/src/c2p_report.hxx:14-271): status codes.
enum RepStatus {
  REP_SUCCESS = 0,
  REP_INVALID_DETG,
  REP_NEG_BSQR,
  REP_NANS_IN_CONS,
  REP_RANGE_RHO,
  REP_RANGE_EPS,
  REP_SPEED_LIMIT,
  REP_RANGE_YE,
  REP_B_LIMIT,
  REP_ROOT_FAIL_CONV,
  REP_ROOT_FAIL_BRACKET,
  REP_PREP_ROOT_FAIL_CONV,
  REP_PREP_ROOT_FAIL_BRACKET,
  REP_NOT_SET,
  // (engine only) the fast pass left the cell to the full cascade
  REP_DEFER
};
struct Report {
  int status = REP_NOT_SET;
  bool adjust_cons = false;
  bool set_atmo = false;
  int iters = 0;
  AXB_HD bool failed() const { return status != REP_SUCCESS; }
  AXB_HD void fail(int s) {
    status = s;
    set_atmo = false;
    adjust_cons = true;
  }
};

struct Atmo {
  double rho, eps, ye, press, temp, entropy, rho_cut;
  AXB_HD void set(Prim &pv) const {
    pv.rho = rho;
    pv.eps = eps;
    pv.Ye = ye;
    pv.press = press;
    pv.temperature = temp;
    pv.entropy = entropy;
    pv.vel[0] = pv.vel[1] = pv.vel[2] = 0.0;
    pv.w_lor = 1.0;
    pv.E[0] = pv.E[1] = pv.E[2] = 0.0;
  }
  AXB_HD void set(Prim &pv, Cons &cv, const sym3 &g) const {
    set(pv);
    const double sqrt_detg = sqrt(det3(g));
    cv.dens = sqrt_detg * rho;
    cv.mom[0] = cv.mom[1] = cv.mom[2] = 0.0;
    cv.DYe = cv.dens * ye;
    cv.DEnt = cv.dens * entropy;
    double Bl[3];
    lower3(g, pv.Bvec, Bl);
    const double Bsq = dot3(pv.Bvec, Bl);
    cv.tau = cv.dens * eps + 0.5 * sqrt_detg * Bsq;
  }
};

struct C2PParams {
  int maxIter, minbits; // minbits = int(|ln tol| / ln 2), computed on the host
  double tol, tolerance_0, alp_thresh, cons_error, vw_lim, w_lim, v_lim,
      Bsq_lim, rho_BH, eps_BH, vwlim_BH;
  int ye_lenient, use_zprim, use_temp, use_press_atmo;
};

// cons_vars::from_prim (Con2PrimFactory/src/cons.hxx:48-91)
AXB_HD void cons_from_prim(Cons &cv, const Prim &pv, const sym3 &g) {
  const double sqrt_detg = sqrt(det3(g));
  double v_low[3], B_low[3];
  lower3(g, pv.vel, v_low);
  const double W = pv.w_lor;
  lower3(g, pv.Bvec, B_low);
  const double bst = W * dot3(pv.Bvec, v_low);
  double b_low[3];
  for (int i = 0; i < 3; ++i)
    b_low[i] = B_low[i] / W + bst * v_low[i];
  const double bs2 = (dot3(pv.Bvec, B_low) + bst * bst) / (W * W);
  cv.dens = sqrt_detg * pv.rho * W;
  const double hW2 = W * W * (pv.rho * (1.0 + pv.eps) + pv.press + bs2);
  for (int i = 0; i < 3; ++i)
    cv.mom[i] = sqrt_detg * (hW2 * v_low[i] - bst * b_low[i]);
  cv.tau = sqrt_detg * (hW2 - (pv.press + 0.5 * bs2) - bst * bst) - cv.dens;
  for (int i = 0; i < 3; ++i)
    cv.dBvec[i] = sqrt_detg * pv.Bvec[i];
  cv.DYe = cv.dens * pv.Ye;
  cv.DEnt = cv.dens * pv.entropy;
}

// c2p::cons_floors_and_ceilings (Con2PrimFactory/src/c2p.hxx:330-369)
AXB_HD void cons_floors(Cons &cv, const sym3 &glo) {
  const double spatial_detg = det3(glo);
  const double sqrt_detg = sqrt(spatial_detg);
  const sym3 gup = inv3(glo, spatial_detg);
  double B_low[3];
  lower3(glo, cv.dBvec, B_low);
  const double BsqL = dot3(B_low, cv.dBvec);
  const double tau_lim = 0.5 * BsqL / sqrt_detg;
  if (cv.tau <= tau_lim)
    cv.tau = tau_lim;
  double mom_up[3];
  lower3(gup, cv.mom, mom_up);
  const double mom2L = dot3(cv.mom, mom_up);
  const double slim = cv.dens + cv.tau;
  const double slim2 = slim * slim;
  if (mom2L > slim2) {
    const double f = sqrt(slim2 / mom2L);
    for (int i = 0; i < 3; ++i)
      cv.mom[i] = cv.mom[i] * f;
  }
}

// c2p::prims_floors_and_ceilings (Con2PrimFactory/src/c2p.hxx:86-216)
template <class EOS>
AXB_HD void prims_floors(const EOS &eos, const C2PParams &cp, const Atmo &atmo,
                         Prim &pv, const Cons &cv, const sym3 &glo,
                         Report &rep) {
  bool recomp = false;
  if (pv.Ye < eos.rgye.min) {
    pv.Ye = eos.rgye.min;
    rep.adjust_cons = true;
    recomp = true;
  }
  if (pv.Ye > eos.rgye.max) {
    pv.Ye = eos.rgye.max;
    rep.adjust_cons = true;
    recomp = true;
  }
  double v_low[3];
  lower3(glo, pv.vel, v_low);
  const double vsq_Sol = dot3(v_low, pv.vel);
  const double sol_v = sqrt(vsq_Sol);
  if (sol_v > cp.v_lim) {
    pv.rho = cv.dens / cp.w_lim;
    const double f = cp.v_lim / sol_v;
    for (int i = 0; i < 3; ++i)
      pv.vel[i] *= f;
    pv.w_lor = cp.w_lim;
    rep.adjust_cons = true;
    if (cp.use_temp) {
      recomp = true;
    } else {
      recomp = false;
      pv.eps = eos.eps_from_valid_rho_press_ye(pv.rho, pv.press, pv.Ye);
      pv.temperature = eos.temp_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
      pv.entropy = eos.kappa_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    }
  }
  if (pv.rho > eos.rgrho.max) {
    pv.rho = eos.rgrho.max;
    rep.adjust_cons = true;
    if (cp.use_temp) {
      recomp = true;
    } else {
      recomp = false;
      pv.eps = eos.eps_from_valid_rho_press_ye(pv.rho, pv.press, pv.Ye);
      pv.temperature = eos.temp_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
      pv.entropy = eos.kappa_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    }
  }
  if (pv.temperature > eos.rgtemp.max) {
    pv.temperature = eos.rgtemp.max;
    recomp = true;
    rep.adjust_cons = true;
  }
  if (cp.use_press_atmo) {
    if (pv.press < atmo.press) {
      pv.press = atmo.press;
      pv.eps = eos.eps_from_valid_rho_press_ye(pv.rho, pv.press, pv.Ye);
      pv.temperature = eos.temp_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
      pv.entropy = eos.kappa_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
      recomp = false;
      rep.adjust_cons = true;
    }
  } else {
    if (pv.temperature < atmo.temp) {
      pv.temperature = atmo.temp;
      recomp = true;
      rep.adjust_cons = true;
    }
  }
  if (recomp) {
    pv.eps = eos.eps_from_valid_rho_temp_ye(pv.rho, pv.temperature, pv.Ye);
    pv.press = eos.press_from_valid_rho_temp_ye(pv.rho, pv.temperature, pv.Ye);
    pv.entropy = eos.kappa_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
  }
}

// c2p::bh_interior (Con2PrimFactory/src/c2p.hxx:218-328)
template <bool LIMITING, class EOS>
AXB_HD void bh_interior(const EOS &eos, const C2PParams &cp, const Atmo &atmo,
                        Prim &pv, Cons &cv, const sym3 &glo) {
  const double wlim_BH = sqrt(1.0 + cp.vwlim_BH * cp.vwlim_BH);
  const double vlim_BH = cp.vwlim_BH / wlim_BH;
  if (LIMITING) {
    bool recomp = false;
    if (pv.rho > cp.rho_BH) {
      pv.rho = cp.rho_BH;
      recomp = true;
    }
    if (pv.eps > cp.eps_BH) {
      pv.eps = cp.eps_BH;
      recomp = true;
    }
    const double sol_v = sqrt((pv.w_lor * pv.w_lor - 1.0)) / pv.w_lor;
    if (sol_v > vlim_BH) {
      const double f = vlim_BH / sol_v;
      for (int i = 0; i < 3; ++i)
        pv.vel[i] *= f;
      pv.w_lor = wlim_BH;
      recomp = true;
    }
    if (recomp) {
      pv.temperature = eos.temp_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
      pv.press = eos.press_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
      pv.entropy = eos.kappa_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
      cons_from_prim(cv, pv, glo);
    }
  } else {
    pv.rho = cp.rho_BH;
    pv.eps = cp.eps_BH;
    pv.Ye = atmo.ye;
    pv.temperature = eos.temp_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    pv.press = eos.press_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    pv.entropy = eos.kappa_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    const double spatial_detg = det3(glo);
    const sym3 gup = inv3(glo, spatial_detg);
    const double Z_loc = (pv.rho * (1.0 + pv.eps) + pv.press) * wlim_BH * wlim_BH;
    double B_low[3];
    lower3(glo, pv.Bvec, B_low);
    const double Bsq = dot3(B_low, pv.Bvec);
    const double sq_detg = sqrt(spatial_detg);
    double mom_low[3], mom_up[3];
    for (int i = 0; i < 3; ++i)
      mom_low[i] = cv.mom[i] / sq_detg;
    lower3(gup, mom_low, mom_up);
    const double Ssq_old = dot3(mom_low, mom_up);
    const double S_old = sqrt(Ssq_old) + 1e-50;
    const double BiSi_old = dot3(mom_low, pv.Bvec);
    const double BiEsi = BiSi_old / S_old;
    const double Ssq_new =
        ((Z_loc + Bsq) * (Z_loc + Bsq) * vlim_BH * vlim_BH) /
        (1.0 + BiEsi * BiEsi * (2.0 * Z_loc + Bsq) / (Z_loc * Z_loc));
    const double S_new = sqrt(Ssq_new);
    for (int i = 0; i < 3; ++i) {
      mom_low[i] *= S_new / S_old;
      mom_up[i] *= S_new / S_old;
    }
    for (int i = 0; i < 3; ++i) {
      pv.vel[i] = mom_up[i] / (Z_loc + Bsq);
      pv.vel[i] += BiEsi * S_new * pv.Bvec[i] / (Z_loc * (Z_loc + Bsq));
    }
    pv.w_lor = wlim_BH;
    cons_from_prim(cv, pv, glo);
  }
}

// Velocity from (Z, W): shared tail of WZ2Prim (c2p_2DNoble.hxx:198-256)
// and xPalenzuelaToPrim (c2p_1DPalenzuela.hxx:188-244).
AXB_HD void vel_from_Z(double Z_Sol, double W_Sol, double Bsq, double BiSi,
                       bool use_zprim, Prim &pv, const Cons &cv,
                       const sym3 &gup, const sym3 &glo) {
  if (use_zprim) {
    double z[3];
    for (int i = 0; i < 3; ++i) {
      const double gm = gup(i, 0) * cv.mom[0] + gup(i, 1) * cv.mom[1] +
                        gup(i, 2) * cv.mom[2];
      z[i] = W_Sol * gm / (Z_Sol + Bsq);
      z[i] += W_Sol * BiSi * cv.dBvec[i] / (Z_Sol * (Z_Sol + Bsq));
    }
    double zd[3];
    lower3(glo, z, zd);
    const double Zsq = z[0] * zd[0] + z[1] * zd[1] + z[2] * zd[2];
    const double SafeLor = sqrt(1.0 + Zsq);
    for (int i = 0; i < 3; ++i)
      pv.vel[i] = z[i] / SafeLor;
    pv.w_lor = SafeLor;
  } else {
    // 1/(Z (Z+B^2)) and 1/(Z+B^2) from one division (last-ulp differences)
    const double iZZB = 1.0 / (Z_Sol * (Z_Sol + Bsq));
    const double iZB = Z_Sol * iZZB;
    for (int i = 0; i < 3; ++i) {
      const double gm = gup(i, 0) * cv.mom[0] + gup(i, 1) * cv.mom[1] +
                        gup(i, 2) * cv.mom[2];
      pv.vel[i] = gm * iZB;
      pv.vel[i] += BiSi * cv.dBvec[i] * iZZB;
    }
    pv.w_lor = W_Sol;
  }
}

// E = gup . (B x v)  (calc_cross_product then calc_contraction)
AXB_HD void set_E(Prim &pv, const sym3 &gup) {
  const double El[3] = {pv.Bvec[1] * pv.vel[2] - pv.Bvec[2] * pv.vel[1],
                        pv.Bvec[2] * pv.vel[0] - pv.Bvec[0] * pv.vel[2],
                        pv.Bvec[0] * pv.vel[1] - pv.Bvec[1] * pv.vel[0]};
  lower3(gup, El, pv.E);
}

// ---------------------------------------------------------------------------
// Noble 2D (c2p_2DNoble::solve, c2p_2DNoble.hxx:275-594).  The ideal-gas
// pressure P(Z, v^2) = (Z(1-v^2) - D sqrt(1-v^2)) (Gamma-1)/Gamma closes the
// system, as in the reference; `gamma` is the EOS's Gamma.
// Seeds (rho, eps, Ye, vel) come in pv_seeds; `zguess` >= 0 replaces the
// Z seed and `vsqguess` in [0,1) the v^2 seed (learned initial guess).
// ---------------------------------------------------------------------------
template <class EOS>
AXB_HD void noble_solve(const EOS &eos, const C2PParams &cp, const Atmo &atmo,
                        double gamma, double Zmin, Prim &pv, Prim &pv_seeds,
                        Cons &cv, const sym3 &glo, Report &rep,
                        double zguess = -1.0, double vsqguess = -1.0) {
  rep.iters = 0;
  rep.adjust_cons = false;
  rep.set_atmo = false;
  rep.status = REP_SUCCESS;
  const double spatial_detg = det3(glo);
  const double sqrt_detg = sqrt(spatial_detg);
  const bool minor1 = glo.xx > 0.0;
  const bool minor2 = glo.xx * glo.yy - glo.xy * glo.xy > 0.0;
  const bool minor3 = spatial_detg > 0.0;
  if (!(minor1 && minor2 && minor3)) {
    rep.fail(REP_INVALID_DETG);
    pv.set_nan();
    cv.set_nan();
    return;
  }
  const sym3 gup = inv3(glo, spatial_detg);
  cv.unscale(sqrt_detg);
  for (int i = 0; i < 3; ++i)
    pv_seeds.Bvec[i] = cv.dBvec[i];
  double mom_up[3];
  lower3(gup, cv.mom, mom_up);
  const double Ssq = dot3(cv.mom, mom_up);
  double B_low[3];
  lower3(glo, pv_seeds.Bvec, B_low);
  const double Bsq = dot3(B_low, pv_seeds.Bvec);
  const double BiSi = dot3(cv.mom, pv_seeds.Bvec);
  double vsq_seed;
  if (cp.use_zprim) {
    double z[3], zl[3];
    for (int i = 0; i < 3; ++i)
      z[i] = pv_seeds.vel[i] * pv_seeds.w_lor;
    lower3(glo, z, zl);
    const double zsq = dot3(zl, z);
    const double w = sqrt(1. + zsq);
    pv_seeds.w_lor = w;
    vsq_seed = fmin(zsq / w / w, 1. - 1.e-15);
  } else {
    double vl[3];
    lower3(glo, pv_seeds.vel, vl);
    const double vsq = dot3(vl, pv_seeds.vel);
    pv_seeds.w_lor = 1. / sqrt(1. - vsq);
    vsq_seed = vsq;
  }
  if (!isfinite(cv.dens) || !isfinite(Ssq) || !isfinite(Bsq) || !isfinite(BiSi) ||
      !isfinite(cv.DYe) || !isfinite(cv.DEnt)) {
    rep.fail(REP_NANS_IN_CONS);
    pv.set_nan();
    cv.set_nan();
    return;
  }
  if (Bsq > cp.Bsq_lim) {
    rep.fail(REP_B_LIMIT);
    pv.set_nan();
    cv.set_nan();
    return;
  }
  pv_seeds.rho = cv.dens / pv_seeds.w_lor;
  double eps_last = fmax(pv_seeds.eps, atmo.eps);
  pv_seeds.press = eos.press_from_valid_rho_eps_ye(pv_seeds.rho, eps_last, pv_seeds.Ye);
  const double Z_Seed = (pv_seeds.rho + eps_last * pv_seeds.rho + pv_seeds.press) *
                        pv_seeds.w_lor * pv_seeds.w_lor;
  double x0 = fabs(Z_Seed), x1 = vsq_seed;
  if (zguess >= 0.0) {
    x0 = zguess;
    x1 = vsqguess;
  }
  double xo0 = x0;
  constexpr double dv = (1. - 1.e-10);
  double errx = 1., df = 1., f = 1.;
  if (x1 < 0.0)
    x1 = 0.0;
  else if (x1 >= 1.0)
    x1 = dv;
  if (x0 <= 0.0)
    x0 = fabs(x0) + Zmin;
  else if (x0 > 1e20)
    x0 = xo0;
  const double gfac = (gamma - 1.0);
  int k;
  for (k = 1; k <= cp.maxIter; k++) {
    const double Z = x0;
    const double invZ = 1.0 / Z;
    const double Vsq = x1;
    const double Sdotn = -(cv.tau + cv.dens);
    const double p_tmp = ((Z * (1.0 - Vsq) - cv.dens * sqrt(1.0 - Vsq)) * gfac / (gamma));
    const double dPdvsq = ((-Z + cv.dens / (2.0 * sqrt(1.0 - Vsq))) * gfac / gamma);
    const double dPdZ = ((1.0 - Vsq) * gfac / gamma);
    const double fj00 = -2 * (Vsq + BiSi * BiSi * invZ * invZ * invZ) * (Bsq + Z);
    const double fj01 = -(Bsq + Z) * (Bsq + Z);
    const double fj10 = -1.0 + dPdZ - BiSi * BiSi * invZ * invZ * invZ;
    const double fj11 = -0.5 * Bsq + dPdvsq;
    const double r0 = Ssq - Vsq * (Bsq + Z) * (Bsq + Z) +
                      BiSi * BiSi * invZ * invZ * (Bsq + Z + Z);
    const double r1 = -Sdotn - 0.5 * Bsq * (1.0 + Vsq) +
                      0.5 * BiSi * BiSi * invZ * invZ - Z + p_tmp;
    const double detjac =
        (Bsq + Z) * (fj10 * (Bsq + Z) +
                     (Bsq - 2.0 * dPdvsq) * (BiSi * BiSi * invZ * invZ + Vsq * Z) * invZ);
    const double detjac_inv = 1.0 / detjac;
    const double dx0 = -(fj11 * r0 - fj01 * r1) * detjac_inv;
    const double dx1 = -(-fj10 * r0 + fj00 * r1) * detjac_inv;
    df = -r0 * r0 - r1 * r1;
    f = -0.5 * (df);
    errx = 0.;
    xo0 = x0;
    x0 += dx0;
    x1 += dx1;
    if (x1 < 0.0)
      x1 = 0.0;
    else if (x1 >= 1.0)
      x1 = dv;
    if (x0 <= 0.0)
      x0 = fabs(x0) + Zmin;
    else if (x0 > 1e20)
      x0 = xo0;
    errx = (x0 == 0.) ? fabs(dx0) : fabs(dx0 / x0);
    if (fabs(errx) <= cp.tol)
      break;
  }
  rep.iters = k;
  if (fabs(errx) > cp.tol) {
    rep.fail(REP_ROOT_FAIL_CONV);
    cv.scale(sqrt_detg);
    return;
  }
  if (!isfinite(f) || !isfinite(df))
    rep.fail(REP_ROOT_FAIL_BRACKET);
  // WZ2Prim (c2p_2DNoble.hxx:192-273)
  {
    const double Z_Sol = x0, vsq_Sol = x1;
    const double W_Sol = 1.0 / sqrt(1.0 - vsq_Sol);
    pv.rho = cv.dens / W_Sol;
    vel_from_Z(Z_Sol, W_Sol, Bsq, BiSi, cp.use_zprim, pv, cv, gup, glo);
    pv.eps = (Z_Sol / pv.w_lor / pv.w_lor / pv.rho - 1.0) / gamma;
    pv.Ye = cv.DYe / cv.dens;
    pv.press = eos.press_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    pv.temperature = eos.temp_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    pv.entropy = eos.kappa_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    for (int i = 0; i < 3; ++i)
      pv.Bvec[i] = cv.dBvec[i];
    set_E(pv, gup);
  }
  if (pv.rho <= 0.0) {
    rep.fail(REP_RANGE_RHO);
    cv.scale(sqrt_detg);
    return;
  }
  if (pv.eps <= 0.0) {
    rep.fail(REP_RANGE_EPS);
    cv.scale(sqrt_detg);
    return;
  }
  cv.DEnt = cv.dens * pv.entropy;
  if (pv.rho < atmo.rho_cut) {
    rep.status = REP_SUCCESS;
    rep.set_atmo = true;
    rep.adjust_cons = true;
    atmo.set(pv, cv, glo);
    return;
  }
  prims_floors(eos, cp, atmo, pv, cv, glo, rep);
  if (rep.adjust_cons)
    cons_from_prim(cv, pv, glo);
  else
    cv.scale(sqrt_detg);
}

// Brent's method as a resumable state: brent_init handles the bracket's
// degenerate cases (a root at an end, no sign change), brent_step does one
// iteration of the loop; brent_bracket runs them to completion.
struct BrentState {
  double a, b, c, d, fa, fb, fc;
  int iters;
  bool mflag;
};
// true: the result (lo, hi) is final without an iteration
AXB_HD bool brent_init(BrentState &st, double a, double b, double fa, double fb, double &lo,
                       double &hi) {
  st.iters = 0;
  if (fa == 0) {
    lo = hi = a;
    return true;
  }
  if (fb == 0) {
    lo = hi = b;
    return true;
  }
  if (fa * fb > 0) {
    lo = fmin(a, b);
    hi = fmax(a, b);
    return true;
  }
  if (fabs(fa) < fabs(fb)) {
    double t = a; a = b; b = t;
    t = fa; fa = fb; fb = t;
  }
  st.a = a;
  st.b = b;
  st.fa = fa;
  st.fb = fb;
  st.c = a;
  st.fc = fa;
  st.d = a;
  st.mflag = true;
  return false;
}
// One pass of the loop; true when (lo, hi) is final.  `eps` = 2^-minbits.
template <class F>
AXB_HD bool brent_step(BrentState &st, const F &f, double eps, int maxiters, double &lo,
                       double &hi) {
  double a = st.a, b = st.b, c = st.c, d = st.d, fa = st.fa, fb = st.fb, fc = st.fc;
  if (st.iters >= maxiters || fabs(b - a) <= eps * fmin(fabs(a), fabs(b))) {
    lo = fmin(a, b);
    hi = fmax(a, b);
    return true;
  }
  ++st.iters;
  double s;
  if (fa != fc && fb != fc) {
    // inverse quadratic interpolation over one common denominator
    // (fa-fb)(fa-fc)(fb-fc) instead of three (last-ulp differences)
    const double dab = fa - fb, dac = fa - fc, dbc = fb - fc;
    s = (a * fb * fc * dbc - b * fa * fc * dac + c * fa * fb * dab) / (dab * dac * dbc);
  } else {
    s = b - fb * (b - a) / (fb - fa);
  }
  const double delta = eps * fabs(b);
  const double q = (3 * a + b) / 4;
  const bool mflag = st.mflag;
  const bool out_of_range = !((s > fmin(q, b)) && (s < fmax(q, b)));
  if (out_of_range || (mflag && fabs(s - b) >= fabs(b - c) / 2) ||
      (!mflag && fabs(s - b) >= fabs(c - d) / 2) || (mflag && fabs(b - c) < delta) ||
      (!mflag && fabs(c - d) < delta)) {
    s = (a + b) / 2;
    st.mflag = true;
  } else {
    st.mflag = false;
  }
  const double fs = f(s);
  d = c;
  c = b;
  fc = fb;
  if (fa * fs < 0) {
    b = s;
    fb = fs;
  } else {
    a = s;
    fa = fs;
  }
  if (fabs(fa) < fabs(fb)) {
    double t = a; a = b; b = t;
    t = fa; fa = fb; fb = t;
  }
  st.a = a;
  st.b = b;
  st.c = c;
  st.d = d;
  st.fa = fa;
  st.fb = fb;
  st.fc = fc;
  if (fb == 0) {
    lo = hi = b;
    return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Brent's bracketing root finder with the contract of CarpetX's Algo::brent
// as used at c2p_1DPalenzuela.hxx:380-417: returns a bracket (lo, hi) of a
// sign change, stopping once |hi-lo| <= 2^-minbits min(|lo|,|hi|) or after
// maxiters iterations.  Same steps as the host stand-in used to build the
// reference checker (inverse quadratic / secant / bisection, R. P. Brent
// 1973).
// ---------------------------------------------------------------------------
// `fa0`, `fb0` are f(a) and f(b), which the caller has evaluated already
// (the reference evaluates them again inside its brent; f is deterministic,
// so the values are the same).
template <class F>
AXB_HD void brent_bracket(const F &f, double a, double b, double fa0, double fb0,
                          int minbits, int maxiters, int &iters, double &lo, double &hi) {
  const double eps = ldexp(1.0, -minbits);
  BrentState st;
  if (brent_init(st, a, b, fa0, fb0, lo, hi)) {
    iters = 0;
    return;
  }
  while (!brent_step(st, f, eps, maxiters, lo, hi)) {
  }
  iters = st.iters;
}

// Palenzuela invariants (c2p_1DPalenzuela.hxx:150-153,267-270), plus the
// loop-invariant Ye of the root function
struct PalQRST {
  double q, r, s, t, ye;
};

// Root function of the Palenzuela scheme (c2p_1DPalenzuela.hxx:264-303).
// W^-2 is clamped as in the reference; W = (W^-2)^(-1/2) is taken as rsqrt
// instead of pow and 1/W as W^-2 W, 1/x and 1/(x (x+s)) come from one
// division, and P/rho comes from the EOS without a division (last-ulp
// differences; the bracket search converges to the same tolerance).
template <class EOS>
AXB_HD double pal_froot(const EOS &eos, const C2PParams &cp, const Atmo &atmo,
                        const PalQRST &k, double x, const Cons &cv) {
  const double xs = x + k.s;
  const double ixxs = 1.0 / (x * xs); // 1/(x (x+s)); 1/x = (x+s)/(x (x+s))
  const double ix = xs * ixxs;
  double Wminus2 = 1.0 - (x * x * k.r + (2.0 * x + k.s) * k.t * k.t) * (ixxs * ixxs);
  Wminus2 = fmin(fmax(Wminus2, 1e-10), 1);
  const double W_loc = rsqrt(Wminus2);
  const double iW = Wminus2 * W_loc;
  const double rho_loc = cv.dens * iW;
  const double Ye_loc = k.ye;
  double eps_loc = W_loc - 1.0 + (1.0 - W_loc * W_loc) * x * iW +
                   W_loc * (k.q - k.s + 0.5 * k.t * k.t * (ix * ix) + 0.5 * k.s * Wminus2);
  if (cp.use_temp) {
    eps_loc = fmax(eps_loc, atmo.eps);
    eps_loc = fmin(eps_loc, eos.rgeps.max);
  }
  return (x - (1.0 + eps_loc + eos.press_over_rho(rho_loc, eps_loc, Ye_loc)) * W_loc);
}

// Palenzuela 1D (c2p_1DPalenzuela::solve, c2p_1DPalenzuela.hxx:306-556).
// `xlo`/`xhi` > 0 narrow the initial bracket (learned initial guess); the
// reference bracket is used when they are negative or do not bracket.
// FAST: the common path only -- every failure, and a bracket that did not
// converge (which needs the conservative-variable check), returns REP_DEFER
// before anything else, so the caller can hand the cell to the full cascade.
template <class EOS, bool FAST = false>
AXB_HD void palenzuela_solve(const EOS &eos, const C2PParams &cp, const Atmo &atmo,
                             Prim &pv, Cons &cv, const sym3 &glo, Report &rep,
                             double xlo = -1.0, double xhi = -1.0) {
  rep.iters = 0;
  rep.adjust_cons = false;
  rep.set_atmo = false;
  rep.status = REP_SUCCESS;
  const double spatial_detg = det3(glo);
  const double sqrt_detg = sqrt(spatial_detg);
  const bool minor1 = glo.xx > 0.0;
  const bool minor2 = glo.xx * glo.yy - glo.xy * glo.xy > 0.0;
  const bool minor3 = spatial_detg > 0.0;
  if (!(minor1 && minor2 && minor3)) {
    if constexpr (FAST) {
      rep.status = REP_DEFER;
      return;
    }
    rep.fail(REP_INVALID_DETG);
    pv.set_nan();
    cv.set_nan();
    return;
  }
  const sym3 gup = inv3(glo, spatial_detg);
  cv.unscale(sqrt_detg);
  double mom_up[3];
  lower3(gup, cv.mom, mom_up);
  const double Ssq = cv.mom[0] * mom_up[0] + cv.mom[1] * mom_up[1] + cv.mom[2] * mom_up[2];
  double B_low[3];
  lower3(glo, cv.dBvec, B_low);
  const double Bsq = dot3(B_low, cv.dBvec);
  const double BiSi =
      cv.dBvec[0] * cv.mom[0] + cv.dBvec[1] * cv.mom[1] + cv.dBvec[2] * cv.mom[2];
  if (!isfinite(cv.dens) || !isfinite(Ssq) || !isfinite(Bsq) || !isfinite(BiSi) ||
      !isfinite(cv.DYe) || !isfinite(cv.DEnt)) {
    if constexpr (FAST) {
      rep.status = REP_DEFER;
      return;
    }
    rep.fail(REP_NANS_IN_CONS);
    pv.set_nan();
    cv.set_nan();
    return;
  }
  if (Bsq > cp.Bsq_lim) {
    if constexpr (FAST) {
      rep.status = REP_DEFER;
      return;
    }
    rep.fail(REP_B_LIMIT);
    pv.set_nan();
    cv.set_nan();
    return;
  }
  // the invariants as products with 1/dens and dens^(-1/2) = rsqrt(dens)
  // instead of five divisions and a pow (last-ulp differences)
  const double idens = 1.0 / cv.dens;
  PalQRST k;
  k.q = cv.tau * idens;
  k.r = Ssq * (idens * idens);
  k.s = Bsq * idens;
  k.t = BiSi * (idens * rsqrt(cv.dens));
  k.ye = cv.DYe * idens;
  const double qP = k.q;
  const double sP = k.s;
  double a = fmax(1e-10, 1.0 + qP - sP);
  double b = 2.0 + 2.0 * qP - sP;
  auto fn = [&](double x) { return pal_froot(eos, cp, atmo, k, x, cv); };
  bool narrowed = false;
  double fa = 0.0, fb = 0.0;
  if (xlo > 0.0 && xhi > xlo) {
    const double flo = fn(xlo), fhi = fn(xhi);
    if (flo * fhi < 0) {
      a = xlo;
      b = xhi;
      fa = flo;
      fb = fhi;
      narrowed = true;
    }
  }
  if (!narrowed) {
    fa = fn(a);
    fb = fn(b);
    if (fa * fb > 0) {
      b = 3.0 + 3.0 * qP - 1.5 * sP;
      fb = fn(b);
    }
  }
  double r0, r1;
  brent_bracket(fn, a, b, fa, fb, cp.minbits, cp.maxIter, rep.iters, r0, r1);
  const bool converged = !(fabs(r0 - r1) > cp.tolerance_0 * fmin(fabs(r0), fabs(r1)));
  if constexpr (FAST) {
    if (!converged) {
      rep.status = REP_DEFER;
      return;
    }
  }
  const double x_sol = 0.5 * (r0 + r1);
  // xPalenzuelaToPrim (c2p_1DPalenzuela.hxx:142-258); W = rsqrt(W^-2)
  // instead of pow, the divisions by W and W^2 as products with W^-1 and
  // W^-2 (last-ulp differences)
  {
    // 1/x^2 = (x+s)^2 / (x^2 (x+s)^2): one division
    const double xs2 = (x_sol + k.s) * (x_sol + k.s);
    const double iden = 1.0 / (x_sol * x_sol * xs2);
    double Wminus2 = 1.0 - (x_sol * x_sol * k.r + (2.0 * x_sol + k.s) * k.t * k.t) * iden;
    Wminus2 = fmin(fmax(Wminus2, 1e-10), 1);
    const double W_sol = rsqrt(Wminus2);
    const double iW = Wminus2 * W_sol;
    pv.rho = cv.dens * iW;
    pv.eps = W_sol - 1.0 + (1.0 - W_sol * W_sol) * x_sol * iW +
             W_sol * (k.q - k.s + 0.5 * k.t * k.t * (xs2 * iden) + 0.5 * k.s * Wminus2);
    if (cp.use_temp) {
      pv.eps = fmax(pv.eps, atmo.eps);
      pv.eps = fmin(pv.eps, eos.rgeps.max);
    }
    const double Z_Sol = x_sol * pv.rho * W_sol;
    vel_from_Z(Z_Sol, W_sol, Bsq, BiSi, cp.use_zprim, pv, cv, gup, glo);
    pv.Ye = cv.DYe / cv.dens;
    pv.press = eos.press_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    pv.temperature = eos.temp_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    pv.entropy = eos.kappa_from_valid_rho_eps_ye(pv.rho, pv.eps, pv.Ye);
    for (int i = 0; i < 3; ++i)
      pv.Bvec[i] = cv.dBvec[i];
    set_E(pv, gup);
  }
  if constexpr (FAST) {
    if (!(pv.rho > 0.0) || !(pv.eps > 0.0)) {
      rep.status = REP_DEFER;
      return;
    }
  }
  if (pv.rho <= 0.0) {
    rep.fail(REP_RANGE_RHO);
    cv.scale(sqrt_detg);
    return;
  }
  if (pv.eps <= 0.0) {
    rep.fail(REP_RANGE_EPS);
    cv.scale(sqrt_detg);
    return;
  }
  if (!FAST && !converged) {
    Cons ck;
    cons_from_prim(ck, pv, glo);
    ck.unscale(sqrt_detg);
    const double small = 1e-50;
    const double e0 = sq((ck.dens - cv.dens) / (cv.dens + small));
    const double e1 = sq((ck.mom[0] - cv.mom[0]) / (cv.mom[0] + small));
    const double e2 = sq((ck.mom[1] - cv.mom[1]) / (cv.mom[1] + small));
    const double e3 = sq((ck.mom[2] - cv.mom[2]) / (cv.mom[2] + small));
    const double e4 = sq((ck.tau - cv.tau) / (cv.tau + small));
    // std::max over an initializer list keeps the first of equal maxima and
    // never selects a NaN unless it is the first element
    double m = e0;
    if (m < e1) m = e1;
    if (m < e2) m = e2;
    if (m < e3) m = e3;
    if (m < e4) m = e4;
    const double max_error = sqrt(m);
    if (max_error > cp.cons_error) {
      rep.fail(REP_ROOT_FAIL_CONV);
      cv.scale(sqrt_detg);
      return;
    }
  }
  cv.DEnt = cv.dens * pv.entropy;
  if (pv.rho < atmo.rho_cut) {
    rep.status = REP_SUCCESS;
    rep.set_atmo = true;
    rep.adjust_cons = true;
    atmo.set(pv, cv, glo);
    return;
  }
  prims_floors(eos, cp, atmo, pv, cv, glo, rep);
  if (rep.adjust_cons)
    cons_from_prim(cv, pv, glo);
  else
    cv.scale(sqrt_detg);
}

// Root function of the entropy scheme (c2p_1DEntropy.hxx:262-303, Appendix
// A.4 of arXiv:1112.0568): with rho = x, p and eps from the conserved
// entropy, W = rho h Lorentz^2 (A60), S_f^2 (A61), rho (A62); returns
// x - rho.  Written as the reference writes it (a backup scheme).
template <class EOS>
AXB_HD double ent_froot(const EOS &eos, double Ssq, double Bsq, double BiSi, double x,
                        const Cons &cv) {
  const double ent_loc = cv.DEnt / cv.dens;
  const double ye_loc = cv.DYe / cv.dens;
  const double press_loc = eos.press_from_valid_rho_kappa_ye(x, ent_loc, ye_loc);
  const double eps_loc = eos.eps_from_valid_rho_kappa_ye(x, ent_loc, ye_loc);
  const double lor_loc = cv.dens / x;
  const double h_loc = (1.0 + eps_loc + press_loc / x);
  const double W = x * h_loc * lor_loc * lor_loc;
  const double Sfsq = (W * W * Ssq + BiSi * BiSi * (Bsq + 2.0 * W)) / ((W + Bsq) * (W + Bsq));
  const double rho = cv.dens / sqrt(1.0 + Sfsq / (cv.dens * cv.dens * h_loc * h_loc));
  return x - rho;
}

// Entropy 1D (c2p_1DEntropy::solve, c2p_1DEntropy.hxx:306-469): Brent on
// rho in [D / sqrt(1 + S^2 / D^2), D] (A59), primitives from the conserved
// entropy (xEntropyToPrim, :143-225), tau recomputed from them.  The
// conservative-variable check of an unconverged bracket omits tau and
// rejects at max_error >= cons_error, as the reference does.
template <class EOS>
AXB_HD void entropy_solve(const EOS &eos, const C2PParams &cp, const Atmo &atmo, Prim &pv,
                          Cons &cv, const sym3 &glo, Report &rep) {
  rep.iters = 0;
  rep.adjust_cons = false;
  rep.set_atmo = false;
  rep.status = REP_SUCCESS;
  const double spatial_detg = det3(glo);
  const double sqrt_detg = sqrt(spatial_detg);
  const bool minor1 = glo.xx > 0.0;
  const bool minor2 = glo.xx * glo.yy - glo.xy * glo.xy > 0.0;
  const bool minor3 = spatial_detg > 0.0;
  if (!(minor1 && minor2 && minor3)) {
    rep.fail(REP_INVALID_DETG);
    pv.set_nan();
    cv.set_nan();
    return;
  }
  const sym3 gup = inv3(glo, spatial_detg);
  cv.unscale(sqrt_detg);
  double mom_up[3];
  lower3(gup, cv.mom, mom_up);
  const double Ssq = cv.mom[0] * mom_up[0] + cv.mom[1] * mom_up[1] + cv.mom[2] * mom_up[2];
  double B_low[3];
  lower3(glo, cv.dBvec, B_low);
  const double Bsq = dot3(B_low, cv.dBvec);
  const double BiSi =
      cv.dBvec[0] * cv.mom[0] + cv.dBvec[1] * cv.mom[1] + cv.dBvec[2] * cv.mom[2];
  if (!isfinite(cv.dens) || !isfinite(Ssq) || !isfinite(Bsq) || !isfinite(BiSi) ||
      !isfinite(cv.DYe) || !isfinite(cv.DEnt)) {
    rep.fail(REP_NANS_IN_CONS);
    pv.set_nan();
    cv.set_nan();
    return;
  }
  if (Bsq > cp.Bsq_lim) {
    rep.fail(REP_B_LIMIT);
    pv.set_nan();
    cv.set_nan();
    return;
  }
  const double a = cv.dens / sqrt(1.0 + Ssq / (cv.dens * cv.dens));
  const double b = cv.dens;
  auto fn = [&](double x) { return ent_froot(eos, Ssq, Bsq, BiSi, x, cv); };
  double r0, r1;
  brent_bracket(fn, a, b, fn(a), fn(b), cp.minbits, cp.maxIter, rep.iters, r0, r1);
  const double x_sol = 0.5 * (r0 + r1);
  // xEntropyToPrim
  pv.rho = x_sol;
  pv.entropy = cv.DEnt / cv.dens;
  pv.Ye = cv.DYe / cv.dens;
  pv.w_lor = cv.dens / x_sol;
  pv.press = eos.press_from_valid_rho_kappa_ye(x_sol, pv.entropy, pv.Ye);
  pv.eps = eos.eps_from_valid_rho_kappa_ye(x_sol, pv.entropy, pv.Ye);
  pv.temperature = eos.temp_from_valid_rho_eps_ye(x_sol, pv.eps, pv.Ye);
  const double Z_Sol = (x_sol + pv.eps * x_sol + pv.press) * pv.w_lor * pv.w_lor;
  vel_from_Z(Z_Sol, pv.w_lor, Bsq, BiSi, cp.use_zprim, pv, cv, gup, glo);
  for (int i = 0; i < 3; ++i)
    pv.Bvec[i] = cv.dBvec[i];
  set_E(pv, gup);
  if (pv.rho <= 0.0) {
    rep.fail(REP_RANGE_RHO);
    cv.scale(sqrt_detg);
    return;
  }
  if (fabs(r0 - r1) > cp.tolerance_0 * fmin(fabs(r0), fabs(r1))) {
    Cons ck;
    cons_from_prim(ck, pv, glo);
    ck.unscale(sqrt_detg);
    const double small = 1e-50;
    const double e0 = sq((ck.dens - cv.dens) / (cv.dens + small));
    const double e1 = sq((ck.mom[0] - cv.mom[0]) / (cv.mom[0] + small));
    const double e2 = sq((ck.mom[1] - cv.mom[1]) / (cv.mom[1] + small));
    const double e3 = sq((ck.mom[2] - cv.mom[2]) / (cv.mom[2] + small));
    double m = e0; // std::max over an initializer list (first of equal maxima)
    if (m < e1) m = e1;
    if (m < e2) m = e2;
    if (m < e3) m = e3;
    if (sqrt(m) >= cp.cons_error) {
      rep.fail(REP_ROOT_FAIL_CONV);
      cv.scale(sqrt_detg);
      return;
    }
  }
  // tau from the recovered primitives (undensitised)
  double v_low[3];
  lower3(glo, pv.vel, v_low);
  const double bst = pv.w_lor * dot3(pv.Bvec, v_low);
  const double bs2 = (Bsq + bst * bst) / (pv.w_lor * pv.w_lor);
  cv.tau = (pv.w_lor * pv.w_lor * (pv.rho * (1.0 + pv.eps) + pv.press + bs2) -
            (pv.press + 0.5 * bs2) - bst * bst) -
           cv.dens;
  if (pv.rho < atmo.rho_cut) {
    rep.status = REP_SUCCESS;
    rep.set_atmo = true;
    rep.adjust_cons = true;
    atmo.set(pv, cv, glo);
    return;
  }
  prims_floors(eos, cp, atmo, pv, cv, glo, rep);
  if (rep.adjust_cons)
    cons_from_prim(cv, pv, glo);
  else
    cv.scale(sqrt_detg);
}

} // namespace axb
