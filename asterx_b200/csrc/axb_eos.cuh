// EOSX equations of state on the device.
//
//   EosIdeal   EOSX/src/eos_3p_idealgas/eos_3p_idealgas.hxx:115-229
//   EosTab     EOSX/src/eos_3p_tabulated3d/eos_3p_tabulated3d.hxx:197-350
//              with the trilinear interpolator of
//              EOSX/src/utils/eos_linear_interp_ND.hxx:50-206 and Brent's
//              zero finder EOSX/src/utils/eos_brent.hxx:7-170
//
// Both keep the reference's call shape: eps is passed by reference and the
// tabulated queries may clamp it in place, as the reference does.
#pragma once

#include <cmath>

#include "axb_common.cuh"

namespace axb {

struct Range {
  double min, max;
};

struct EosIdeal {
  double gamma, gm1, inv_gamma, temp_over_eps;
  Range rgrho, rgye, rgtemp, rgeps;
  // rho^(1-gamma) of the entropy without pow for the common adiabatic
  // indices (set by make_ideal): 3 -> gamma = 4/3, rcbrt(rho); 5 -> 5/3,
  // rcbrt(rho)^2; 2 -> gamma = 2, 1/rho; 0 -> pow (last-ulp differences)
  int kappa_root;

  static constexpr bool kTabulated = false;

  AXB_HD double press_from_valid_rho_eps_ye(double rho, double &eps, double) const {
    return gm1 * rho * eps;
  }
  // P / rho without the division (the root functions of the recovery)
  AXB_HD double press_over_rho(double, double &eps, double) const { return gm1 * eps; }
  AXB_HD double eps_from_valid_rho_press_ye(double rho, double press, double) const {
    return press / (rho * gm1);
  }
  AXB_HD double csnd_from_valid_rho_eps_ye(double, double &eps, double) const {
    return sqrt(gm1 * eps / (eps + inv_gamma));
  }
  // the square of csnd_from_valid_rho_eps_ye without the square root
  AXB_HD double csnd2_from_valid_rho_eps_ye(double, double &eps, double) const {
    return gm1 * eps / (eps + inv_gamma);
  }
  AXB_HD double temp_from_valid_rho_eps_ye(double, double &eps, double) const {
    return temp_over_eps * eps;
  }
  AXB_HD double eps_from_valid_rho_temp_ye(double, double temp, double) const {
    return temp / temp_over_eps;
  }
  AXB_HD double press_from_valid_rho_temp_ye(double rho, double temp, double ye) const {
    double eps = eps_from_valid_rho_temp_ye(rho, temp, ye);
    return press_from_valid_rho_eps_ye(rho, eps, ye);
  }
  // p = kappa rho^Gamma and eps = kappa rho^(Gamma-1) / (Gamma-1) of the
  // evolved entropy (eos_3p_idealgas.hxx:201-215), with pow as there: the
  // entropy recovery's root function, not on a hot path
  AXB_HD double press_from_valid_rho_kappa_ye(double rho, double kappa, double) const {
    return kappa * pow(rho, gamma);
  }
  AXB_HD double eps_from_valid_rho_kappa_ye(double rho, double kappa, double) const {
    return kappa * pow(rho, gamma - 1.0) / (gamma - 1.0);
  }
  AXB_HD double kappa_from_valid_rho_eps_ye(double rho, double &eps, double) const {
    double r;
    if (kappa_root == 3) {
      r = rcbrt(rho);
    } else if (kappa_root == 5) {
      r = rcbrt(rho);
      r *= r;
    } else if (kappa_root == 2) {
      r = 1.0 / rho;
    } else {
      r = pow(rho, 1.0 - gamma);
    }
    return (gamma - 1.0) * eps * r;
  }
};

// Host-side construction mirroring eos_3p_idealgas::init
// (eos_3p_idealgas.hxx:124-142).
inline EosIdeal make_ideal(double gamma, double umass, Range rgeps, Range rgrho,
                           Range rgye) {
  EosIdeal e;
  e.gamma = gamma;
  e.gm1 = gamma - 1;
  e.inv_gamma = 1 / gamma;
  e.rgeps = rgeps;
  if (gamma > 2)
    e.rgeps.max = std::fmin(e.rgeps.max, 1 / (gamma * (gamma - 2)));
  e.rgrho = rgrho;
  e.rgye = rgye;
  e.temp_over_eps = e.gm1 * umass;
  const double expo = 1 - gamma;
  e.kappa_root = std::fabs(expo + 1.0 / 3) < 1e-14   ? 3
                 : std::fabs(expo + 2.0 / 3) < 1e-14 ? 5
                 : expo == -1.0                      ? 2
                                                     : 0;
  e.rgtemp = Range{e.temp_over_eps * e.rgeps.min, e.temp_over_eps * e.rgeps.max};
  return e;
}

// 1-parameter polytrope, only used for a cold atmosphere
// (EOSX/src/eos_1p_polytropic/eos_1p_polytropic.hxx:57-90).
struct EosPoly {
  double poly_k, poly_gamma, n, np1, invn, rho_p;
  AXB_HD double gm1_from_valid_rho(double rho) const {
    return np1 * pow(rho / rho_p, invn);
  }
  AXB_HD double sed_from_valid_gm1(double gm1) const { return gm1 / poly_gamma; }
};
inline EosPoly make_poly(double poly_gamma, double poly_k) {
  EosPoly p;
  p.poly_k = poly_k;
  p.poly_gamma = poly_gamma;
  p.n = 1.0 / (poly_gamma - 1.0);
  p.np1 = p.n + 1;
  p.invn = 1.0 / p.n;
  p.rho_p = std::pow(poly_k, -p.n);
  return p;
}

} // namespace axb
