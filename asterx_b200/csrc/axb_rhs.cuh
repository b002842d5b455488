// Face physics and the RHS kernels of the engine (AsterX_RHSGroup:
// AsterX_Fluxes + AsterX_SourceTerms + AsterX_RHS).
//
// Kernels (one launch each per box, all FP64):
//   k_flux_pass<DIR>  reconstruct-once + face physics + Riemann flux along
//                     one direction, marching a pencil segment per thread,
//                     with the flux divergence carried in registers
//                     (AsterX/src/fluxes.cxx:216-795, rhs.cxx:107-114,188-207)
//   k_sources         geometric source terms (AsterX/src/source.cxx:20-168)
//   k_aux             vertex auxiliaries F, Fbeta, G (fluxes.cxx:798-826)
//   k_ct_psi          edge E from the face B fluxes (flux-CT), A and Psi RHS
//                     (rhs.cxx:116-186,209-252)
#pragma once

#include "axb_common.cuh"
#include "axb_eos.cuh"
#include "axb_recon.cuh"

namespace axb {

enum { V_DENS = 0, V_MOMX, V_MOMY, V_MOMZ, V_TAU, V_DYE, V_DENT, NHYDRO };

struct RhsArgs {
  BoxDev b;
  const double *rho, *vel[3], *eps, *press, *Ye, *entropy, *Bvec[3];
  // the thermodynamic variable reconstructed with rho, entropy and Ye:
  // temperature when rec_temp, else pressure (fluxes.cxx:257-355)
  const double *temperature, *thermo;
  int rec_temp;
  // the velocity-like variable reconstructed at the faces (recon_type,
  // fluxes.cxx:396-505): vel^i (v_vec), zvec^i = W v^i (z_vec) or
  // svec^i = rho h W^2 v^i (s_vec)
  const double *recv[3];
  int recvar;
  const double *dBstag[3];
  const double *alp, *beta[3], *g[6], *K[6];
  const double *Avec[3], *Psi;
  double *acc[NHYDRO];
  double *rhs[NHYDRO];
  double *bflux[6]; // fxBy fxBz fyBx fyBz fzBx fzBy
  // upwind CT face data (fluxes.cxx:776-794), per face direction d:
  // uct[4d] = vtilde^{d+1}, uct[4d+1] = vtilde^{d+2} (upwind-averaged),
  // uct[4d+2] = amax, uct[4d+3] = amin; written when use_uct
  double *uct[12];
  int use_uct;
  // transverse ghost layers the flux passes cover: 1 (the edge field of
  // flux CT needs one), 3 with upwind CT (its reconstructions to the edges
  // reach three faces out); the kernels take it as a template constant
  int text;
  int recon_method; // reconstruction of the upwind-CT edge values
  double *aux[7];   // Fx Fy Fz Fbetax Fbetay Fbetaz G
  double *Arhs[3], *Psi_rhs;
  // The stage update fused into the group (axb_substep): with fuse_stage
  // the z flux pass and the CT kernel write
  //   U_k <- st_alpha U_n + st_beta U_k + st_gdt RHS
  // for the 11 evolved variables (dens, mom, tau, DYe, DEnt, Avec, Psi; U_k
  // updated in place) instead of storing the RHS grid functions
  int fuse_stage;
  double st_alpha, st_beta, st_gdt;
  const double *st_un[11];
  double *st_uk[11];
  ReconParams rp;
  int recon_lo, flux_type, gauge, fd_order, write_bflux;
  double lorenz_damp_fac;
  DevStatus *status;
};

// Fast magnetosonic speeds of one face state (eigenvalues.hxx:19-79): the
// roots of a2 l^2 + a1 l + a0 = 0 divided by the lapse, lam_p with +sqrt
// and lam_m with -sqrt (the reference lists each twice).  One reciprocal of
// 2 a2 alp instead of the two divisions (last-ulp differences).
AXB_HD void fast_speeds(double alp, double beta, double uinv, double vdir, double rho,
                        double cs2, double W, double h, double bsq, double &lam_p,
                        double &lam_m) {
  const double a0 = (bsq + cs2 * h * rho) * (sq(beta) - sq(alp) * uinv) -
                    (-1 + cs2) * h * rho * sq(beta - alp * vdir) * sq(W);
  const double a1 = 2 * beta * (bsq + cs2 * h * rho) -
                    2 * (-1 + cs2) * h * rho * (beta - alp * vdir) * sq(W);
  const double a2 = bsq + h * rho * (cs2 + sq(W) - cs2 * sq(W));
  double det = sq(a1) - 4 * a2 * a0;
  if (det < 0)
    det = 0;
  const double sd = sqrt(det);
  const double i2a2alp = 1 / (2 * a2 * alp);
  lam_p = (-a1 + sd) * i2a2alp;
  lam_m = (-a1 - sd) * i2a2alp;
}

// Riemann fluxes of one variable (AsterX/src/fluxes.hxx:20-49) from the
// bounding speeds cmax = max(0, speeds) and cmin = min(0, speeds):
// HLLE with the reciprocal icpm = 1 / (cmax - cmin) (a product instead of
// the division), LxF with ch = max(cmax, -cmin) = max |speed|.
// Every operation is rounded on its own (no multiply-add contraction): the
// contraction choices depend on the surrounding kernel, and the single-box
// and batched passes must give a face the same bits.
AXB_HD double hlle_flux(double cmax, double cmin, double icpm, double uL, double uR,
                        double fL, double fR) {
  return mul_rn(add_rn(add_rn(mul_rn(cmax, fL), -mul_rn(cmin, fR)),
                       mul_rn(mul_rn(cmax, cmin), add_rn(uR, -uL))),
                icpm);
}
AXB_HD double laxf_flux(double ch, double uL, double uR, double fL, double fR) {
  return mul_rn(0.5, add_rn(add_rn(fL, fR), -mul_rn(ch, add_rn(uR, -uL))));
}

// The stage combine U_k <- alpha U_n + beta U_k + gdt RHS with an explicit
// rounding order, so that the fused and the separate stage update give the
// same bits.
AXB_D double stage_combine(double alpha, double un, double beta, double uk, double gdt,
                           double rhs) {
  return fma(gdt, rhs, fma(beta, uk, alpha * un));
}

// ---------------------------------------------------------------------------
// face metric: v2f averages of the vertex metric (AsterUtils aster_interp.hxx
// :68-80), determinant, sqrt, and the (dir,dir) element of the inverse
// ---------------------------------------------------------------------------
struct FaceMetric {
  double alp, beta[3];
  sym3 g;
  double detg, sqrtg, isqrtg, uinv;
};

template <int DIR>
AXB_D double avg_v2f(const double *__restrict__ f, long long I, long long s1,
                     long long s2) {
  double a = 0.0;
  a += __ldg(f + I);
  a += __ldg(f + I + s1);
  a += __ldg(f + I + s2);
  a += __ldg(f + I + s1 + s2);
  return a / 4.0;
}

template <int DIR>
AXB_D FaceMetric face_metric(const RhsArgs &a, long long I) {
  constexpr int D1 = (DIR + 1) % 3, D2 = (DIR + 2) % 3;
  const long long s1 = a.b.stride(D1), s2 = a.b.stride(D2);
  FaceMetric m;
  m.alp = avg_v2f<DIR>(a.alp, I, s1, s2);
  for (int i = 0; i < 3; ++i)
    m.beta[i] = avg_v2f<DIR>(a.beta[i], I, s1, s2);
  m.g.xx = avg_v2f<DIR>(a.g[0], I, s1, s2);
  m.g.xy = avg_v2f<DIR>(a.g[1], I, s1, s2);
  m.g.xz = avg_v2f<DIR>(a.g[2], I, s1, s2);
  m.g.yy = avg_v2f<DIR>(a.g[3], I, s1, s2);
  m.g.yz = avg_v2f<DIR>(a.g[4], I, s1, s2);
  m.g.zz = avg_v2f<DIR>(a.g[5], I, s1, s2);
  m.detg = det3(m.g);
  // sqrt(detg), 1/sqrt(detg) and 1/detg from one rsqrt instead of a square
  // root and two divisions (last-ulp differences)
  m.isqrtg = rsqrt(m.detg);
  m.sqrtg = m.detg * m.isqrtg;
  // (dir,dir) element of calc_inv(g, detg)
  const double idet = m.isqrtg * m.isqrtg;
  if (DIR == 0)
    m.uinv = (m.g.yy * m.g.zz - m.g.yz * m.g.yz) * idet;
  else if (DIR == 1)
    m.uinv = (m.g.xx * m.g.zz - m.g.xz * m.g.xz) * idet;
  else
    m.uinv = (m.g.xx * m.g.yy - m.g.xy * m.g.xy) * idet;
  return m;
}

// Reconstructed primitive state on one side of a face.  r[] order:
//   0 rho, 1 entropy, 2 Ye, 3 press or temperature, 4 vx, 5 vy, 6 vz,
//   7 B_{dir+1}, 8 B_{dir+2}
enum { R_RHO = 0, R_ENT, R_YE, R_PRESS, R_VX, R_VY, R_VZ, R_B1, R_B2, NREC };

struct SideOut {
  double U[10], F[10]; // conserved and flux: dens momx momy momz tau DYe DEnt Bx By Bz
  double lam_p, lam_m; // the two distinct fast speeds of this side
  double vt1, vt2;     // vtilde^{dir+1}, vtilde^{dir+2} (upwind CT)
};

// Per-side physics of CalcFlux (fluxes.cxx:357-654).
// With rec_temp, r[R_PRESS] holds the reconstructed temperature and eps and
// press come from (rho, T, Ye) (fluxes.cxx:297-304); otherwise eps comes
// from (rho, press, Ye) (:346-353; the temperature computed there is unused
// and only the tabulated EOS, which cannot take this route, would clamp eps).
// r[R_VX..R_VZ] hold the reconstructed vel^i, zvec^i or svec^i (recvar):
// W and v^i follow from them as in fluxes.cxx:396-505.
// UCT: also the transverse vtilde components (upwind CT)
template <int DIR, bool UCT, class EOS>
AXB_D void side_physics(const FaceMetric &m, const double *r, double Bdir,
                        const EOS &eos, int rec_temp, int recvar, SideOut &o) {
  constexpr int D1 = (DIR + 1) % 3, D2 = (DIR + 2) % 3;
  const double rho = r[R_RHO], ent = r[R_ENT], ye = r[R_YE];
  double eps, press;
  if (rec_temp) {
    eps = eos.eps_from_valid_rho_temp_ye(rho, r[R_PRESS], ye);
    press = eos.press_from_valid_rho_temp_ye(rho, r[R_PRESS], ye);
  } else {
    press = r[R_PRESS];
    eps = eos.eps_from_valid_rho_press_ye(rho, press, ye);
  }
  double B[3];
  B[DIR] = Bdir;
  B[D1] = r[R_B1];
  B[D2] = r[R_B2];
  double vel[3], vlow[3], W, iW;
  if (recvar == AXB_RECVAR_V) {
    vel[0] = r[R_VX];
    vel[1] = r[R_VY];
    vel[2] = r[R_VZ];
    lower3(m.g, vel, vlow);
    // W = rsqrt(1 - v^2) and 1/W = (1 - v^2) W, used in four places as a
    // product (last-ulp differences from the reference's divisions by W)
    const double omv2 = 1 - dot3(vlow, vel);
    W = rsqrt(omv2);
    iW = omv2 * W;
  } else {
    // z_vec: W = sqrt(1 + z_i z^i), v^i = z^i / W (fluxes.cxx:453-463);
    // s_vec: W^2 = 1/2 + sqrt(1/4 + s_i s^i / (rho h)^2),
    // v^i = s^i / (W^2 rho h) (:492-504).  The divisions by W (and rho h)
    // are products with one reciprocal here, and for z_vec 1/W is one rsqrt
    // with W = (1 + z^2) / W (last-ulp differences).
    const double q[3] = {r[R_VX], r[R_VY], r[R_VZ]};
    double qlow[3];
    lower3(m.g, q, qlow);
    const double qq = dot3(qlow, q);
    double f;
    if (recvar == AXB_RECVAR_Z) {
      const double opz2 = 1 + qq;
      iW = rsqrt(opz2);
      W = opz2 * iW;
      f = iW;
    } else {
      const double rhoh = rho + rho * eps + press;
      W = sqrt(0.5 + sqrt(0.25 + qq / rhoh / rhoh));
      iW = 1 / W;
      f = iW * iW / rhoh;
    }
    for (int i = 0; i < 3; ++i) {
      vel[i] = q[i] * f;
      vlow[i] = qlow[i] * f;
    }
  }
  double vt[3];
  for (int i = 0; i < 3; ++i)
    vt[i] = m.alp * vel[i] - m.beta[i];
  if constexpr (UCT) {
    o.vt1 = vt[D1];
    o.vt2 = vt[D2];
  }
  const double alp_b0 = W * dot3(B, vlow);
  double Blow[3];
  lower3(m.g, B, Blow);
  const double B2 = dot3(B, Blow);
  double blow[3];
  for (int i = 0; i < 3; ++i)
    blow[i] = Blow[i] * iW + alp_b0 * vlow[i];
  const double bsq = (B2 + sq(alp_b0)) * sq(iW);
  // cs^2 as the product of two sound-speed queries (fluxes.cxx:556-560); the
  // first may clamp eps in place (tabulated), and only then can the second
  // differ from the first
  double cs2, h;
  if constexpr (EOS::kTabulated) {
    const double eps_in = eps;
    const double cs = eos.csnd_from_valid_rho_eps_ye(rho, eps, ye);
    cs2 = cs * (!(eps == eps_in) ? eos.csnd_from_valid_rho_eps_ye(rho, eps, ye) : cs);
    h = 1 + eps + press / rho;
  } else {
    // ideal gas: cs^2 without the square root, P/rho without the division
    // (last-ulp differences)
    cs2 = eos.csnd2_from_valid_rho_eps_ye(rho, eps, ye);
    h = 1 + eps + eos.press_over_rho(rho, eps, ye);
  }
  const double dens = m.sqrtg * rho * W;
  const double DEnt = m.sqrtg * rho * W * ent;
  const double dhW = dens * h * W;
  const double dhWp = dhW + m.sqrtg * (sq(alp_b0) + B2);
  const double ppm = press + 0.5 * bsq;
  const double vtd = vt[DIR];
  const double alp_sqrtg = m.alp * m.sqrtg;
  const double BoW = B[DIR] * iW;
  o.U[0] = dens;
  o.F[0] = dens * vtd;
  for (int j = 0; j < 3; ++j) {
    const double mom = dhWp * vlow[j] - m.sqrtg * alp_b0 * blow[j];
    o.U[1 + j] = mom;
    o.F[1 + j] = mom * vtd + alp_sqrtg * (ppm * (j == DIR ? 1.0 : 0.0) - blow[j] * BoW);
  }
  const double tau = dhW - dens + m.sqrtg * (B2 - ppm);
  o.U[4] = tau;
  o.F[4] = tau * vtd + alp_sqrtg * (ppm * vel[DIR] - alp_b0 * BoW);
  const double DYe = dens * ye;
  o.U[5] = DYe;
  o.F[5] = DYe * vtd;
  o.U[6] = DEnt;
  o.F[6] = DEnt * vtd;
  double Bt[3];
  for (int i = 0; i < 3; ++i)
    Bt[i] = m.sqrtg * B[i];
  const double E0 = Bt[1] * vt[2] - Bt[2] * vt[1];
  const double E1 = Bt[2] * vt[0] - Bt[0] * vt[2];
  const double E2 = Bt[0] * vt[1] - Bt[1] * vt[0];
  o.U[7] = Bt[0];
  o.U[8] = Bt[1];
  o.U[9] = Bt[2];
  // flux(Btilde) = unit_dir x E (fluxes.cxx:650-654)
  if (DIR == 0) {
    o.F[7] = 0.0;
    o.F[8] = -E2;
    o.F[9] = E1;
  } else if (DIR == 1) {
    o.F[7] = E2;
    o.F[8] = 0.0;
    o.F[9] = -E0;
  } else {
    o.F[7] = -E1;
    o.F[8] = E0;
    o.F[9] = 0.0;
  }
  fast_speeds(m.alp, m.beta[DIR], m.uinv, vel[DIR], rho, cs2, W, h, bsq, o.lam_p, o.lam_m);
}

} // namespace axb
