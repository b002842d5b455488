// Test infrastructure only: the Cactus parameters the reference hot path
// reads (AsterX/param.ccl, ReconX/param.ccl, Con2PrimFactory/param.ccl,
// EOSX/param.ccl), held in one struct that the harness fills.
#ifndef AXREF_SHIM_CCTK_PARAMETERS_H
#define AXREF_SHIM_CCTK_PARAMETERS_H

#include <cctk.h>

struct axref_params_t {
  // keywords
  const char *recon_type, *reconstruction_method, *loworder_method,
      *flux_type, *evolution_eos, *vector_potential_gauge, *c2p_prime,
      *c2p_second;
  // booleans and integers
  CCTK_INT reconstruct_with_temperature, ppm_shock_detection,
      ppm_zone_flattening, use_uct, local_spatial_order, thermal_eos_atmo,
      use_press_atmo, max_iter, use_mask, excise, debug_mode, use_entropy_fix,
      Ye_lenient, use_z, use_temperature, interpolate_failed_c2p,
      tmunu_interp_order;
  // reals
  CCTK_REAL poly_k, poly_gamma, ppm_eta1, ppm_eta2, ppm_eps, ppm_eps_shock,
      ppm_small, ppm_omega1, ppm_omega2, enhanced_ppm_C2, weno_eps, mp5_alpha,
      lorenz_damp_fac, r_atmo, rho_abs_min, n_rho_atmo, p_atmo, n_press_atmo,
      Ye_atmo, t_atmo, n_temp_atmo, atmo_tol, c2p_tol, alp_thresh,
      cons_error_limit, vw_lim, B_lim, rho_BH, eps_BH, vwlim_BH, gl_gamma,
      eps_atmo;
};

extern axref_params_t axref_params;

#define AXREF_P(name) const auto &name = axref_params.name; (void)name;

#define DECLARE_CCTK_PARAMETERS                                                \
  AXREF_P(recon_type) AXREF_P(reconstruction_method) AXREF_P(loworder_method)  \
  AXREF_P(flux_type) AXREF_P(evolution_eos) AXREF_P(vector_potential_gauge)    \
  AXREF_P(c2p_prime) AXREF_P(c2p_second)                                       \
  AXREF_P(reconstruct_with_temperature) AXREF_P(ppm_shock_detection)           \
  AXREF_P(ppm_zone_flattening) AXREF_P(use_uct) AXREF_P(local_spatial_order)   \
  AXREF_P(thermal_eos_atmo) AXREF_P(use_press_atmo) AXREF_P(max_iter)          \
  AXREF_P(use_mask) AXREF_P(excise) AXREF_P(debug_mode)                        \
  AXREF_P(use_entropy_fix) AXREF_P(Ye_lenient) AXREF_P(use_z)                  \
  AXREF_P(use_temperature) AXREF_P(interpolate_failed_c2p)                     \
  AXREF_P(tmunu_interp_order)                                                  \
  AXREF_P(poly_k) AXREF_P(poly_gamma) AXREF_P(ppm_eta1) AXREF_P(ppm_eta2)      \
  AXREF_P(ppm_eps) AXREF_P(ppm_eps_shock) AXREF_P(ppm_small)                   \
  AXREF_P(ppm_omega1) AXREF_P(ppm_omega2) AXREF_P(enhanced_ppm_C2)             \
  AXREF_P(weno_eps) AXREF_P(mp5_alpha) AXREF_P(lorenz_damp_fac)                \
  AXREF_P(r_atmo) AXREF_P(rho_abs_min) AXREF_P(n_rho_atmo) AXREF_P(p_atmo)     \
  AXREF_P(n_press_atmo) AXREF_P(Ye_atmo) AXREF_P(t_atmo) AXREF_P(n_temp_atmo)  \
  AXREF_P(atmo_tol) AXREF_P(c2p_tol) AXREF_P(alp_thresh)                       \
  AXREF_P(cons_error_limit) AXREF_P(vw_lim) AXREF_P(B_lim) AXREF_P(rho_BH)     \
  AXREF_P(eps_BH) AXREF_P(vwlim_BH) AXREF_P(gl_gamma) AXREF_P(eps_atmo)

#endif
