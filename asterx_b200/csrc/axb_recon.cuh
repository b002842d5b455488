// ReconX reconstruction operators, per cell.
//
// Every scheme here produces the two interface values of ONE cell c, its
// lower value (at face c) and its upper value (at face c+1), from the cells
// c-2 .. c+2.  The reference evaluates the same per-cell formulas inside
// ReconX::reconstruct once per face, i.e. twice per cell
// (ReconX/src/ppm.hxx:163-180, wenoz.hxx:104-113, mp5.hxx:79-94); the values
// are identical, so a face's left state is the upper value of cell i-1 and
// its right state the lower value of cell i:
//   ppm        ReconX/src/ppm.hxx:21-161 (Colella & Woodward 1984, with the
//              contact-discontinuity steepening for rho and the optional
//              zone flattening)
//   wenoz      ReconX/src/wenoz.hxx:21-102 (Borges et al. 2008, GRHydro
//              candidate stencils)
//   mp5        ReconX/src/mp5.hxx:24-77 (Suresh & Huynh 1997, alpha, early
//              accept at 1e-10)
//   minmod     ReconX/src/minmod.hxx:13-42
//   monocentral ReconX/src/monocentral.hxx:15-45
//   godunov    ReconX/src/reconstruct.hxx:53-55 (cell value)
#pragma once

#include <cmath>

#include "axb_common.cuh"

namespace axb {

struct ReconParams {
  int ppm_shock_detection, ppm_zone_flattening;
  double poly_k, poly_gamma, ppm_eta1, ppm_eta2, ppm_eps, ppm_eps_shock,
      ppm_small, ppm_omega1, ppm_omega2, weno_eps, mp5_alpha;
};

AXB_HD int sgn_int(double v) { return (0.0 < v) - (v < 0.0); }

AXB_HD double minmod2(double x, double y) {
  // selects only (no branch): 0 for opposite signs, else the smaller
  // magnitude (y on ties), as ReconX's minmod
  const double m = fabs(x) < fabs(y) ? x : y;
  return signbit(x) != signbit(y) ? 0.0 : m;
}

AXB_HD double monocentral2(double x, double y) {
  if (sgn_int(x) != sgn_int(y))
    return 0;
  return sgn_int(x) * fmin(2 * fabs(x), fmin(2 * fabs(y), fabs(x + y) / 2));
}

// Cell values q[0..4] = c-2 .. c+2.  For PPM, pr[0..4] holds the pressure on
// the same cells and vel[1], vel[3] the velocity along the pencil at c-1 and
// c+1 (only read with zone flattening).
struct CellLoUp {
  double lo, up;
};

AXB_HD CellLoUp recon_ppm(const double q[5], const double pr[5],
                          const double vel[5], bool is_rho,
                          const ReconParams &rp) {
  const double gf_Imm = q[0], gf_Im = q[1], gf_I = q[2], gf_Ip = q[3],
               gf_Ipp = q[4];
  const double press_Imm = pr[0], press_Im = pr[1], press_Ip = pr[3],
               press_Ipp = pr[4];
  const double diff_Im = gf_I - gf_Imm;
  const double diff_I = gf_Ip - gf_Im;
  const double diff_Ip = gf_Ipp - gf_I;
  const double delta_Im = 0.5 * diff_Im;
  const double delta_I = 0.5 * diff_I;
  const double delta_Ip = 0.5 * diff_Ip;
  const double f_Im_Imm = 2 * fabs(gf_Im - gf_Imm);
  const double f_I_Im = 2 * fabs(gf_I - gf_Im);
  const double f_Ip_I = 2 * fabs(gf_Ip - gf_I);
  const double f_Ipp_Ip = 2 * fabs(gf_Ipp - gf_Ip);
  const bool ss_Im = ((gf_I - gf_Im) * (gf_Im - gf_Imm) > 0);
  const bool ss_I = ((gf_Ip - gf_I) * (gf_I - gf_Im) > 0);
  const bool ss_Ip = ((gf_Ipp - gf_Ip) * (gf_Ip - gf_I) > 0);
  const double dm_Im =
      ss_Im ? sgn_int(delta_Im) * fmin(fabs(delta_Im), fmin(f_Im_Imm, f_I_Im)) : 0;
  const double dm_I =
      ss_I ? sgn_int(delta_I) * fmin(fabs(delta_I), fmin(f_I_Im, f_Ip_I)) : 0;
  const double dm_Ip =
      ss_Ip ? sgn_int(delta_Ip) * fmin(fabs(delta_Ip), fmin(f_Ip_I, f_Ipp_Ip)) : 0;
  double rc_low = 0.5 * (gf_Im + gf_I) + (1. / 6.) * (dm_Im - dm_I);
  double rc_up = 0.5 * (gf_I + gf_Ip) + (1. / 6.) * (dm_I - dm_Ip);
  const double diff_press_I = press_Ip - press_Im;
  const double min_press_I = fmin(press_Im, press_Ip);
  if (rp.ppm_shock_detection && is_rho) {
    const double k_gamma = rp.poly_k * rp.poly_gamma;
    const bool contact = (k_gamma * fabs(diff_I) * min_press_I >=
                          fabs(diff_press_I) * fmin(gf_Ip, gf_Im));
    if (contact) {
      const double d2_Im = gf_I - 2 * gf_Im + gf_Imm;
      const double d2_Ip = gf_Ipp - 2 * gf_Ip + gf_I;
      const double d2_prod = d2_Im * d2_Ip;
      const bool cond2 =
          (fabs(diff_I) - rp.ppm_eps_shock * fmin(fabs(gf_Ip), fabs(gf_Im))) > 0.;
      const double eta_tilde =
          ((d2_prod < 0) && cond2) ? ((-1. / 6.) * (d2_Ip - d2_Im) / diff_I) : 0;
      const double eta = fmax(0., fmin(rp.ppm_eta1 * (eta_tilde - rp.ppm_eta2), 1.));
      rc_low = (1 - eta) * rc_low + eta * (gf_Im + 0.5 * dm_Im);
      rc_up = (1 - eta) * rc_up + eta * (gf_Ip - 0.5 * dm_Ip);
    }
  }
  if (rp.ppm_zone_flattening) {
    const double w =
        ((fabs(diff_press_I) > rp.ppm_eps * min_press_I) && (vel[1] > vel[3]))
            ? 1.
            : 0;
    const double ft =
        (fabs(press_Ipp - press_Imm) < rp.ppm_small)
            ? 1.0
            : fmax(0., 1. - w * fmax(0., rp.ppm_omega2 *
                                             ((diff_press_I / (press_Ipp - press_Imm)) -
                                              rp.ppm_omega1)));
    const double omf = (1 - ft) * gf_I;
    rc_low = ft * rc_low + omf;
    rc_up = ft * rc_up + omf;
  }
  if ((rc_up - gf_I) * (gf_I - rc_low) <= 0) {
    rc_low = gf_I;
    rc_up = gf_I;
  } else {
    const double d = rc_up - rc_low;
    const double d2 = d * d;
    const double g6 = 6 * d * (gf_I - 0.5 * (rc_low + rc_up));
    if (g6 > d2)
      rc_low = 3 * gf_I - 2 * rc_up;
    else if (g6 < -d2)
      rc_up = 3 * gf_I - 2 * rc_low;
  }
  return {rc_low, rc_up};
}

// 2^-e for a positive normal x = m 2^e (1 <= m < 2): an exact rescaling
AXB_HD double pow2_inv_exponent(double x) {
#ifdef __CUDA_ARCH__
  const long long E = (__double_as_longlong(x) >> 52) & 0x7ff;
  return __longlong_as_double((2046 - E) << 52);
#else
  return std::ldexp(1.0, -std::ilogb(x));
#endif
}

AXB_HD CellLoUp recon_wenoz(const double q[5], double weno_eps) {
  // Same weights and candidate stencils as the reference, with its divisions
  // regrouped into ONE per cell (last-ulp differences).  With
  // d_k = beta_k + eps and P = d0 d1 d2, the unnormalised weight
  // w_k (1 + tau5 / d_k) is w_k n_k / P with n_k = P + tau5 prod_{j != k} d_j;
  // the common 1/P cancels in the normalisation, so both sides' weights (and
  // the 1/6 of the stencils) share one reciprocal of the product of the two
  // weight sums.  The n_k are scaled by an exact power of two that brings P
  // to [1, 2), so n_k ~ 1 + tau5 / d_k as in the reference and the product of
  // the sums stays far from overflow for |values| < 1e50 (eps = 1e-26 bounds
  // d_k below).
  const double a = q[0], b = q[1], c = q[2], d = q[3], e = q[4];
  const double beta0 = (13.0 / 12.0) * sq(a - 2.0 * b + c) +
                       (1.0 / 4.0) * sq(a - 4.0 * b + 3.0 * c);
  const double beta1 =
      (13.0 / 12.0) * sq(b - 2.0 * c + d) + (1.0 / 4.0) * sq(b - d);
  const double beta2 = (13.0 / 12.0) * sq(c - 2.0 * d + e) +
                       (1.0 / 4.0) * sq(3.0 * c - 4.0 * d + e);
  const double tau5 = fabs(beta0 - beta2);
  const double d0 = beta0 + weno_eps, d1 = beta1 + weno_eps, d2 = beta2 + weno_eps;
  const double P = d0 * d1 * d2;
  const double sc = pow2_inv_exponent(P);
  const double Ps = P * sc, ts = tau5 * sc;
  const double aux0 = Ps + ts * (d1 * d2);
  const double aux1 = Ps + ts * (d0 * d2);
  const double aux2 = Ps + ts * (d0 * d1);
  const double w0 = 3.0 / 10.0, w1 = 3.0 / 5.0, w2 = 1.0 / 10.0;
  // minus side (lower value): weights w0, w1, w2; plus side: w2, w1, w0
  const double am0 = w0 * aux0, am1 = w1 * aux1, am2 = w2 * aux2;
  const double ap0 = w2 * aux0, ap1 = w1 * aux1, ap2 = w0 * aux2;
  const double sm = am0 + am1 + am2, sp = ap0 + ap1 + ap2;
  const double rr = 1.0 / (6.0 * sm * sp);
  const double idm6 = sp * rr, idp6 = sm * rr;
  const double var_m = (am2 * (2.0 * e - 7.0 * d + 11.0 * c) +
                        am1 * (-1.0 * d + 5.0 * c + 2.0 * b) +
                        am0 * (2.0 * c + 5.0 * b - 1.0 * a)) *
                       idm6;
  const double var_p = (ap0 * (2.0 * a - 7.0 * b + 11.0 * c) +
                        ap1 * (-1.0 * b + 5.0 * c + 2.0 * d) +
                        ap2 * (2.0 * c + 5.0 * d - 1.0 * e)) *
                       idp6;
  return {var_m, var_p};
}

// Products and sums rounded one by one, never fused into a multiply-add
// (the reference's CPU build rounds every operation as written): for the
// values that feed a branch decision, so that both builds take the same
// branch.
AXB_HD double mul_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
AXB_HD double add_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}

// x / 60, correctly rounded, without a division: q = RN(x r) with
// r = RN(1/60) lies within an ulp of x / 60, so x - 60 q is exact (one FMA),
// and q + (x - 60 q) r (one FMA) is off x / 60 by at most about 2^-53 ulp
// before its rounding.  x / 60 = (x / 4) / 15 is either representable or at
// least 1/30 ulp from the nearest midpoint (15 is odd), so that rounding
// gives the correctly rounded quotient (Markstein's correction step,
// IBM J. Res. Dev. 34(1), 1990; for divisors known in advance, Brisebarre,
// Muller and Raina, IEEE Trans. Comput. 53(8), 2004).  The bounds need x
// and q in the normal range; zeros, subnormals, infinities and NaN take the
// division.
AXB_HD double div60(double x) {
#ifdef __CUDA_ARCH__
  constexpr double r = 1.0 / 60.0;
  const double q = __dmul_rn(x, r);
  const double aq = fabs(q);
  if (!(aq >= 0x1p-960 && aq <= 0x1p1000))
    return x / 60.0;
  const double rem = fma(-q, 60.0, x);
  return fma(rem, r, q);
#else
  return x / 60.0;
#endif
}

#ifndef AXB_MP5_SELECT
#define AXB_MP5_SELECT 1
#endif

// MP5 interface value of the middle cell towards u_p1's side.
AXB_HD double mp5_one(double gf_Imm, double gf_Im, double gf_I, double gf_Ip,
                      double gf_Ipp, double alpha) {
  // ul feeds the early-accept test: the reference's correctly rounded
  // quotient, and its products and sums rounded one by one, left to right
  const double ul = div60(
      add_rn(add_rn(add_rn(add_rn(mul_rn(2, gf_Imm), -mul_rn(13, gf_Im)), mul_rn(47, gf_I)),
                    mul_rn(27, gf_Ip)),
             -mul_rn(3, gf_Ipp)));
  const double deltam = gf_I - gf_Im;
  const double deltap = gf_Ip - gf_I;
  const double ump = gf_I + minmod2(deltap, alpha * deltam);
  const bool accept = mul_rn(ul - gf_I, ul - ump) <= 1.0e-10;
#if !AXB_MP5_SELECT
  if (accept)
    return ul;
#endif
  const double dm = gf_Imm + gf_I - 2 * gf_Im;
  const double d = gf_Im + gf_Ip - 2 * gf_I;
  const double dp = gf_I + gf_Ipp - 2 * gf_Ip;
  const double dmp = minmod2(minmod2(4 * d - dp, 4 * dp - d), minmod2(d, dp));
  const double dmm = minmod2(minmod2(4 * dm - d, 4 * d - dm), minmod2(dm, d));
  const double uul = gf_I + alpha * deltam;
  const double uav = (gf_I + gf_Ip) / 2.0;
  const double umd = uav - dmp / 2.0;
  // (4/3) dmm is the one product here that is not exact: rounded on its
  // own, so no kernel that inlines this contracts it differently
  const double ulc = add_rn(gf_I + deltam / 2.0, mul_rn(4.0 / 3.0, dmm));
  const double umin = fmax(fmin(gf_I, fmin(gf_Ip, umd)), fmin(gf_I, fmin(uul, ulc)));
  const double umax = fmin(fmax(gf_I, fmax(gf_Ip, umd)), fmax(gf_I, fmax(uul, ulc)));
  // median(ul, umin, umax) = ul + minmod(umin - ul, umax - ul)
#if AXB_MP5_SELECT
  // both results computed, the early accept a select: no lane of a warp
  // waits on another lane's limiter branch
  return accept ? ul : ul + minmod2(umin - ul, umax - ul);
#else
  return ul + minmod2(umin - ul, umax - ul);
#endif
}

AXB_HD CellLoUp recon_mp5(const double q[5], double alpha) {
  return {mp5_one(q[4], q[3], q[2], q[1], q[0], alpha),
          mp5_one(q[0], q[1], q[2], q[3], q[4], alpha)};
}

AXB_HD CellLoUp recon_minmod(const double q[5]) {
  const double s = minmod2(q[3] - q[2], q[2] - q[1]) / 2;
  return {q[2] - s, q[2] + s};
}

AXB_HD CellLoUp recon_monocentral(const double q[5]) {
  const double s = monocentral2(q[3] - q[2], q[2] - q[1]) / 2;
  return {q[2] - s, q[2] + s};
}

template <int RECON>
AXB_HD CellLoUp recon_cell(const double q[5], const double pr[5],
                           const double vel[5], bool is_rho,
                           const ReconParams &rp) {
  if constexpr (RECON == AXB_RECON_PPM)
    return recon_ppm(q, pr, vel, is_rho, rp);
  else if constexpr (RECON == AXB_RECON_WENOZ)
    return recon_wenoz(q, rp.weno_eps);
  else if constexpr (RECON == AXB_RECON_MP5)
    return recon_mp5(q, rp.mp5_alpha);
  else if constexpr (RECON == AXB_RECON_MINMOD)
    return recon_minmod(q);
  else if constexpr (RECON == AXB_RECON_MONOCENTRAL)
    return recon_monocentral(q);
  else
    return {q[2], q[2]};
}

// Runtime dispatch for the low-order fallback (Godunov/minmod/monocentral).
AXB_HD CellLoUp recon_cell_lo(int method, const double q[5]) {
  if (method == AXB_RECON_MINMOD)
    return recon_minmod(q);
  if (method == AXB_RECON_MONOCENTRAL)
    return recon_monocentral(q);
  return {q[2], q[2]};
}

} // namespace axb
