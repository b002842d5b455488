// Host-side C wrappers around include/asterx_b200_point.hxx for the CPU test
// of the per-point entry points against the reference functors
// (tests/test_point_api.py).  Test infrastructure: compiled by nvcc as host
// code into tests/_build/libpoint_api.so.
#include "../include/asterx_b200_point.hxx"

#define PT_API extern "C" __attribute__((visibility("default")))

using namespace axb_point;

namespace {
reconstruct_params_t recon_params(const double *r) {
  reconstruct_params_t p;
  p.ppm_shock_detection = int(r[0]);
  p.ppm_zone_flattening = int(r[1]);
  p.poly_k = r[2];
  p.poly_gamma = r[3];
  p.ppm_eta1 = r[4];
  p.ppm_eta2 = r[5];
  p.ppm_eps = r[6];
  p.ppm_eps_shock = r[7];
  p.ppm_small = r[8];
  p.ppm_omega1 = r[9];
  p.ppm_omega2 = r[10];
  p.weno_eps = r[11];
  p.mp5_alpha = r[12];
  return p;
}
} // namespace

// v, pr, vel: the six cells I - 3 .. I + 2 of a pencil; rp[13] as above
PT_API void pt_reconstruct(int method, const double *v, const double *pr, const double *vel,
                           int is_rho, int is_press, const double *rp, double *out) {
  const face_values f = reconstruct(v, 3, 1, reconstruction_t(method), bool(is_rho),
                                    bool(is_press), pr, vel, recon_params(rp));
  out[0] = f[0];
  out[1] = f[1];
}

// in = alp, beta, u, then the pairs vel, rho, cs2, w, h, bsq
PT_API void pt_eigen(const double *in, double *lam) {
  const char_speeds c = eigenvalues(in[0], in[1], in[2], in + 3, in + 5, in + 7, in + 9,
                                    in + 11, in + 13);
  for (int s = 0; s < 2; ++s)
    for (int i = 0; i < 4; ++i)
      lam[4 * s + i] = c.lam[s][i];
}

PT_API double pt_riemann(int flux_type, const double *lam8, double uL, double uR, double fL,
                         double fR) {
  double lam[2][4];
  for (int s = 0; s < 2; ++s)
    for (int i = 0; i < 4; ++i)
      lam[s][i] = lam8[4 * s + i];
  const double var[2] = {uL, uR}, flux[2] = {fL, fR};
  return flux_type == AXB_FLUX_HLLE ? hlle(lam, var, flux) : laxf(lam, var, flux);
}

// prim = rho, vx, vy, vz, eps, press, entropy, Ye, Bx, By, Bz;
// cons = dens, momx, momy, momz, tau, DEnt, DYe, dBx, dBy, dBz
PT_API void pt_prim2con(const double *g6, const double *prim, double *cons) {
  const sym3 g{g6[0], g6[1], g6[2], g6[3], g6[4], g6[5]};
  prim_vars pv;
  pv.set_nan();
  pv.rho = prim[0];
  for (int i = 0; i < 3; ++i) {
    pv.vel[i] = prim[1 + i];
    pv.Bvec[i] = prim[8 + i];
  }
  pv.eps = prim[4];
  pv.press = prim[5];
  pv.entropy = prim[6];
  pv.Ye = prim[7];
  cons_vars cv;
  prim2con(g, pv, cv);
  cons[0] = cv.dens;
  for (int i = 0; i < 3; ++i) {
    cons[1 + i] = cv.mom[i];
    cons[7 + i] = cv.dBvec[i];
  }
  cons[4] = cv.tau;
  cons[5] = cv.DEnt;
  cons[6] = cv.DYe;
}

// One scheme on one cell, the ideal gas eos8 = gamma, umass, eps range,
// rho range, Ye range; c2p14 = max_iter, c2p_tol, alp_thresh,
// cons_error_limit, vw_lim, B_lim, rho_BH, eps_BH, vwlim_BH, Ye_lenient,
// use_z, use_temperature, use_press_atmo; the other arrays as the
// reference checker's ora_c2p_point.
PT_API void pt_c2p(int solver, double *cons, const double *g6, const double *seed,
                   const double *atmo_in, const double *eos8, const double *c2p14,
                   double *prim, int *rep3) {
  const eos_3p_idealgas eos =
      make_idealgas(eos8[0], eos8[1], eos8[2], eos8[3], eos8[4], eos8[5], eos8[6], eos8[7]);
  const atmosphere atmo{atmo_in[0], atmo_in[1], atmo_in[2], atmo_in[3],
                        atmo_in[4], atmo_in[5], atmo_in[6]};
  const sym3 glo{g6[0], g6[1], g6[2], g6[3], g6[4], g6[5]};
  cons_vars cv{cons[0], {cons[1], cons[2], cons[3]}, cons[4], cons[5], cons[6],
               {cons[7], cons[8], cons[9]}};
  prim_vars pv;
  pv.set_nan();
  c2p_report rep;
  const double *q = c2p14;
  if (solver == AXB_C2P_NOBLE) {
    const double sdetg = sqrt(axb::det3(glo));
    prim_vars seeds;
    seeds.set_nan();
    seeds.rho = seed[0];
    seeds.eps = seed[1];
    seeds.Ye = seed[2];
    seeds.press = seed[3];
    seeds.temperature = seed[4];
    seeds.entropy = seed[5];
    for (int i = 0; i < 3; ++i) {
      seeds.vel[i] = seed[6 + i];
      seeds.Bvec[i] = cv.dBvec[i] / sdetg;
    }
    seeds.w_lor = 1.0;
    const c2p_2DNoble s(&eos, atmo, int(q[0]), q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8],
                        q[9] != 0, q[10] != 0, q[11] != 0, q[12] != 0);
    s.solve(&eos, pv, seeds, cv, glo, rep);
  } else {
    const c2p_1DPalenzuela s(&eos, atmo, int(q[0]), q[1], q[2], q[3], q[4], q[5], q[6], q[7],
                             q[8], q[9] != 0, q[10] != 0, q[11] != 0, q[12] != 0);
    s.solve(&eos, pv, cv, glo, rep);
  }
  cons[0] = cv.dens;
  for (int i = 0; i < 3; ++i) {
    cons[1 + i] = cv.mom[i];
    cons[7 + i] = cv.dBvec[i];
  }
  cons[4] = cv.tau;
  cons[5] = cv.DYe;
  cons[6] = cv.DEnt;
  const double pvals[16] = {pv.rho,     pv.eps,     pv.Ye,     pv.press,   pv.temperature,
                            pv.entropy, pv.vel[0],  pv.vel[1], pv.vel[2],  pv.w_lor,
                            pv.Bvec[0], pv.Bvec[1], pv.Bvec[2], pv.E[0],   pv.E[1],
                            pv.E[2]};
  for (int i = 0; i < 16; ++i)
    prim[i] = pvals[i];
  rep3[0] = rep.status;
  rep3[1] = rep.iters;
  rep3[2] = rep.adjust_cons;
}
