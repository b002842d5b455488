/* asterx_b200_point.hxx -- the reference's per-point functions with their
 * signatures, as __host__ __device__ entry points over the engine's own
 * device code (the functions its kernels inline).
 *
 * For a caller that keeps its own loops (a thorn's CCTK_DEVICE lambdas, a
 * unit test on the host) and wants the engine's arithmetic point by point.
 * Compile with nvcc (C++17, --expt-relaxed-constexpr); host code compiled
 * by nvcc can call every function here as well.
 *
 *   reference                                         here
 *   ReconX::reconstruct (ReconX/src/reconstruct.hxx:36-42)       reconstruct
 *   AsterX::eigenvalues (AsterX/src/eigenvalues.hxx:19-24)       eigenvalues
 *   AsterX::laxf, AsterX::hlle (AsterX/src/fluxes.hxx:20-49)     laxf, hlle
 *   AsterX::prim2con (AsterX/src/prim2con.hxx:38-83)             prim2con
 *   c2p_2DNoble::solve (Con2PrimFactory/src/c2p_2DNoble.hxx:275-279)
 *                                                                c2p_2DNoble::solve
 *   c2p_1DPalenzuela::solve (Con2PrimFactory/src/c2p_1DPalenzuela.hxx:306-309)
 *                                                                c2p_1DPalenzuela::solve
 *
 * Differences of form, not of meaning:
 *   - CarpetX's GF3D2 + PointDesc + dir become a pointer, the linear index
 *     of the point (the cell on the plus side of the face, p.I) and the
 *     stride of the direction (p.DI[dir] as an offset);
 *   - Arith vec / smat become plain arrays and axb::sym3;
 *   - the arrays the reference returns by value are small structs.
 * Arithmetic: as the engine's kernels (a reciprocal where the reference
 * divides twice, rsqrt for W): results agree with the reference to the
 * last few ulps; each function names its difference.
 */
#pragma once

#include "../asterx_b200/csrc/axb_c2p.cuh"
#include "../asterx_b200/csrc/axb_eos.cuh"
#include "../asterx_b200/csrc/axb_recon.cuh"
#include "../asterx_b200/csrc/axb_rhs.cuh"
#include "../asterx_b200/csrc/axb_tab.cuh"

namespace axb_point {

using axb::sym3;
using prim_vars = axb::Prim;
using cons_vars = axb::Cons;
using c2p_report = axb::Report;
using atmosphere = axb::Atmo;
using eos_3p_idealgas = axb::EosIdeal;
using eos_3p_tabulated3d = axb::EosTab;

/* ReconX::reconstruction_t, same order (ReconX/src/reconstruct.hxx:25-33). */
enum class reconstruction_t { Godunov, minmod, monocentral, ppm, eppm, wenoz, mp5 };

/* ReconX::reconstruct_params_t: the same members minus enhanced_ppm_C2
 * (eppm is not supported). */
using reconstruct_params_t = axb::ReconParams;

struct face_values {
  double v[2]; /* minus side (upper value of cell I - stride), plus side
                  (lower value of cell I) */
  AXB_HD double operator[](int i) const { return v[i]; }
};

/* ReconX::reconstruct at the face between cells I - stride and I.
 * gf_press and gf_vel_dir (the velocity along the direction) are read by
 * PPM only; gf_is_press only by eppm, which returns NaN here (the engine
 * rejects eppm).  Reads gf_var at I - 3 stride .. I + 2 stride. */
AXB_HD face_values reconstruct(const double *gf_var, long long I, long long stride,
                               reconstruction_t reconstruction, bool gf_is_rho,
                               bool gf_is_press, const double *gf_press,
                               const double *gf_vel_dir,
                               const reconstruct_params_t &rp) {
  (void)gf_is_press;
  double q[6];
  for (int c = 0; c < 6; ++c)
    q[c] = gf_var[I + (c - 3) * stride];
  if (reconstruction == reconstruction_t::Godunov)
    return {{q[2], q[3]}};
  if (reconstruction == reconstruction_t::eppm) {
    const double n = nan("");
    return {{n, n}};
  }
  double pr[6] = {0, 0, 0, 0, 0, 0}, vel[6] = {0, 0, 0, 0, 0, 0};
  if (reconstruction == reconstruction_t::ppm) {
    for (int c = 0; c < 6; ++c) {
      pr[c] = gf_press[I + (c - 3) * stride];
      vel[c] = gf_vel_dir[I + (c - 3) * stride];
    }
  }
  // cell I - stride uses q[0..4], cell I uses q[1..5]
  axb::CellLoUp m, p;
  switch (reconstruction) {
  case reconstruction_t::minmod:
    m = axb::recon_minmod(q);
    p = axb::recon_minmod(q + 1);
    break;
  case reconstruction_t::monocentral:
    m = axb::recon_monocentral(q);
    p = axb::recon_monocentral(q + 1);
    break;
  case reconstruction_t::ppm:
    m = axb::recon_ppm(q, pr, vel, gf_is_rho, rp);
    p = axb::recon_ppm(q + 1, pr + 1, vel + 1, gf_is_rho, rp);
    break;
  case reconstruction_t::wenoz:
    m = axb::recon_wenoz(q, rp.weno_eps);
    p = axb::recon_wenoz(q + 1, rp.weno_eps);
    break;
  default: // mp5
    m = axb::recon_mp5(q, rp.mp5_alpha);
    p = axb::recon_mp5(q + 1, rp.mp5_alpha);
    break;
  }
  return {{m.up, p.lo}};
}

/* AsterX::eigenvalues: lambda[s][0..3] for the minus (s = 0) and plus
 * (s = 1) states; [0] = [1] = the + root, [2] = [3] = the - root. */
struct char_speeds {
  double lam[2][4];
};
AXB_HD char_speeds eigenvalues(double alp_avg, double beta_avg, double u_avg,
                               const double vel[2], const double rho[2],
                               const double cs2[2], const double w_lor[2],
                               const double h[2], const double bsq[2]) {
  char_speeds r;
  for (int s = 0; s < 2; ++s) {
    double lp, lm;
    axb::fast_speeds(alp_avg, beta_avg, u_avg, vel[s], rho[s], cs2[s], w_lor[s], h[s],
                     bsq[s], lp, lm);
    r.lam[s][0] = r.lam[s][1] = lp;
    r.lam[s][2] = r.lam[s][3] = lm;
  }
  return r;
}

namespace detail {
AXB_HD void bounds(const double lam[2][4], double &cmax, double &cmin) {
  cmax = 0.0;
  cmin = 0.0;
  for (int s = 0; s < 2; ++s)
    for (int i = 0; i < 4; ++i) {
      cmax = fmax(cmax, lam[s][i]);
      cmin = fmin(cmin, lam[s][i]);
    }
}
} // namespace detail

/* AsterX::laxf: var = {minus, plus} state, flux = their physical fluxes. */
AXB_HD double laxf(const double lam[2][4], const double var[2], const double flux[2]) {
  double cmax, cmin;
  detail::bounds(lam, cmax, cmin);
  return axb::laxf_flux(fmax(cmax, -cmin), var[0], var[1], flux[0], flux[1]);
}

/* AsterX::hlle (the reciprocal of charmax - charmin times the numerator). */
AXB_HD double hlle(const double lam[2][4], const double var[2], const double flux[2]) {
  double cmax, cmin;
  detail::bounds(lam, cmax, cmin);
  return axb::hlle_flux(cmax, cmin, 1 / (cmax - cmin), var[0], var[1], flux[0], flux[1]);
}

/* AsterX::prim2con: W from the velocity (1 / sqrt(1 - v_i v^i)), then the
 * Valencia map.  pv.w_lor is not read. */
AXB_HD void prim2con(const sym3 &g, const prim_vars &pv, cons_vars &cv) {
  double vlow[3];
  axb::lower3(g, pv.vel, vlow);
  prim_vars q = pv;
  q.w_lor = 1.0 / sqrt(1.0 - axb::dot3(vlow, pv.vel));
  axb::cons_from_prim(cv, q, g);
}

namespace detail {
/* The constructor arguments of both schemes (c2p_2DNoble.hxx:74-79,
 * c2p_1DPalenzuela.hxx:64-69) as the engine's parameter block. */
AXB_HD axb::C2PParams c2p_params(int maxIter, double tol, double alp_thresh,
                                 double consError, double vwlim, double B_lim,
                                 double rho_BH, double eps_BH, double vwlim_BH,
                                 bool ye_len, bool use_z, bool use_temperature,
                                 bool use_pressure_atmo) {
  axb::C2PParams c;
  c.maxIter = maxIter;
  c.tol = tol;
  c.minbits = int(fabs(log(tol)) / log(2.0));
  c.tolerance_0 = ldexp(1.0, -c.minbits);
  c.alp_thresh = alp_thresh;
  c.cons_error = consError;
  c.vw_lim = vwlim;
  c.w_lim = sqrt(1.0 + vwlim * vwlim);
  c.v_lim = vwlim / c.w_lim;
  c.Bsq_lim = B_lim * B_lim;
  c.rho_BH = rho_BH;
  c.eps_BH = eps_BH;
  c.vwlim_BH = vwlim_BH;
  c.ye_lenient = ye_len;
  c.use_zprim = use_z;
  c.use_temp = use_temperature;
  c.use_press_atmo = use_pressure_atmo;
  return c;
}
template <class EOS> AXB_HD double noble_gamma(const EOS &e) {
  if constexpr (EOS::kTabulated)
    return nan("");
  else
    return e.gamma;
}
} // namespace detail

/* Con2PrimFactory's Noble 2D scheme: constructed with the reference's
 * arguments, solve() with its signature. */
struct c2p_2DNoble {
  axb::C2PParams cp;
  atmosphere atmo;
  double gamma, Zmin;
  template <class EOS>
  AXB_HD c2p_2DNoble(const EOS *eos_3p, const atmosphere &atm, int maxIter, double tol,
                     double alp_thresh, double consError, double vwlim, double B_lim,
                     double rho_BH, double eps_BH, double vwlim_BH, bool ye_len,
                     bool use_z, bool use_temperature, bool use_pressure_atmo)
      : cp(detail::c2p_params(maxIter, tol, alp_thresh, consError, vwlim, B_lim, rho_BH,
                              eps_BH, vwlim_BH, ye_len, use_z, use_temperature,
                              use_pressure_atmo)),
        atmo(atm), gamma(detail::noble_gamma(*eos_3p)), Zmin(eos_3p->rgrho.min) {}
  template <class EOS>
  AXB_HD void solve(const EOS *eos_3p, prim_vars &pv, prim_vars &pv_seeds, cons_vars &cv,
                    const sym3 &glo, c2p_report &rep) const {
    axb::noble_solve(*eos_3p, cp, atmo, gamma, Zmin, pv, pv_seeds, cv, glo, rep);
  }
};

/* Con2PrimFactory's Palenzuela 1D scheme. */
struct c2p_1DPalenzuela {
  axb::C2PParams cp;
  atmosphere atmo;
  template <class EOS>
  AXB_HD c2p_1DPalenzuela(const EOS *eos_3p, const atmosphere &atm, int maxIter,
                          double tol, double alp_thresh, double consError, double vwlim,
                          double B_lim, double rho_BH, double eps_BH, double vwlim_BH,
                          bool ye_len, bool use_z, bool use_temperature,
                          bool use_pressure_atmo)
      : cp(detail::c2p_params(maxIter, tol, alp_thresh, consError, vwlim, B_lim, rho_BH,
                              eps_BH, vwlim_BH, ye_len, use_z, use_temperature,
                              use_pressure_atmo)),
        atmo(atm) {
    (void)eos_3p;
  }
  template <class EOS>
  AXB_HD void solve(const EOS *eos_3p, prim_vars &pv, cons_vars &cv, const sym3 &glo,
                    c2p_report &rep) const {
    axb::palenzuela_solve(*eos_3p, cp, atmo, pv, cv, glo, rep);
  }
};

/* eos_3p_idealgas::init (EOSX/src/eos_3p_idealgas/eos_3p_idealgas.hxx:
 * 124-142), host side. */
inline eos_3p_idealgas make_idealgas(double gamma, double umass, double eps_min,
                                     double eps_max, double rho_min, double rho_max,
                                     double ye_min, double ye_max) {
  return axb::make_ideal(gamma, umass, axb::Range{eps_min, eps_max},
                         axb::Range{rho_min, rho_max}, axb::Range{ye_min, ye_max});
}

} // namespace axb_point
