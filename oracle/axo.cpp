// axo.cpp -- the oracle restatement (test infrastructure only).
//
// A CPU restatement, in plain scalar C++, of the reference algorithm of the
// hot path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline load it, as a checker; the product never does.  Every routine
// names the reference file:line it restates, keeps the reference's order of
// floating-point operations (the build uses -ffp-contract=off), and tests
// compare it bit-for-bit with the reference's own sources compiled through
// oracle/refshim.  Summations add terms in index order starting from zero
// (two-index sums: i outer, j inner).
#include "axo.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// state
// ---------------------------------------------------------------------------
const char *kNames[] = {
#define AXO_N(name) #name,
    AXB_GF_LIST(AXO_N)
#undef AXO_N
    // reference-only face data the engine never stores
    "fxdens", "fxmomx", "fxmomy", "fxmomz", "fxtau", "fxDYe", "fxDEnt", "fxBx",
    "fyBy", "fzBz", "fydens", "fymomx", "fymomy", "fymomz", "fytau", "fyDYe",
    "fyDEnt", "fzdens", "fzmomx", "fzmomy", "fzmomz", "fztau", "fzDYe", "fzDEnt"};
constexpr int kNFields = sizeof(kNames) / sizeof(kNames[0]);

struct Box {
  int n[3], ng;
  long long sy, sz;
  double dx[3], xmin[3];
};

Box g_box;
axb_params g_p;
double *g_f[kNFields];
int g_ext_c = 0, g_ext_v = 0;
char g_err[256] = "";

double *F(const char *name) {
  for (int i = 0; i < kNFields; ++i)
    if (!std::strcmp(kNames[i], name))
      return g_f[i];
  return nullptr;
}

struct Fail : std::runtime_error {
  using std::runtime_error::runtime_error;
};

template <class Fn> int guarded(Fn &&fn) {
  try {
    fn();
    return 0;
  } catch (const Fail &e) {
    std::snprintf(g_err, sizeof g_err, "%s", e.what());
    return 1;
  }
}

double *need(const char *name) {
  double *p = F(name);
  if (!p)
    throw Fail(std::string("grid function not bound: ") + name);
  return p;
}

inline long long at(int i, int j, int k) { return i + g_box.sy * j + g_box.sz * k; }
inline long long st(int d) { return d == 0 ? 1 : (d == 1 ? g_box.sy : g_box.sz); }

// Loop over the interior of a centring (1 = cell-centred along the axis),
// widened by ext_c / ext_v (CarpetX loop_int_device semantics).
template <class Fn> void loop(int ci, int cj, int ck, Fn &&fn) {
  const int c[3] = {ci, cj, ck};
  int lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    const int e = c[d] ? g_ext_c : g_ext_v;
    lo[d] = g_box.ng - e;
    hi[d] = g_box.ng + g_box.n[d] + (c[d] ? 0 : 1) + e;
  }
  for (int k = lo[2]; k < hi[2]; ++k)
    for (int j = lo[1]; j < hi[1]; ++j)
      for (int i = lo[0]; i < hi[0]; ++i)
        fn(i, j, k);
}

// ---------------------------------------------------------------------------
// tensor helpers (CarpetX Arith semantics as used by the reference)
// ---------------------------------------------------------------------------
struct Sym {
  double xx, xy, xz, yy, yz, zz;
  double operator()(int i, int j) const {
    if (i > j)
      std::swap(i, j);
    if (i == 0)
      return j == 0 ? xx : (j == 1 ? xy : xz);
    if (i == 1)
      return j == 1 ? yy : yz;
    return zz;
  }
};
double det(const Sym &g) {
  return g.xx * (g.yy * g.zz - g.yz * g.yz) - g.xy * (g.xy * g.zz - g.yz * g.xz) +
         g.xz * (g.xy * g.yz - g.yy * g.xz);
}
Sym inv(const Sym &g, double d) {
  const double id = 1 / d;
  return Sym{(g.yy * g.zz - g.yz * g.yz) * id, (g.xz * g.yz - g.xy * g.zz) * id,
             (g.xy * g.yz - g.xz * g.yy) * id, (g.xx * g.zz - g.xz * g.xz) * id,
             (g.xy * g.xz - g.xx * g.yz) * id, (g.xx * g.yy - g.xy * g.xy) * id};
}
// sum_j g(i,j) v(j), j = 0, 1, 2 from zero
void mul(const Sym &g, const double *v, double *o) {
  for (int i = 0; i < 3; ++i) {
    double s = 0;
    for (int j = 0; j < 3; ++j)
      s += g(i, j) * v[j];
    o[i] = s;
  }
}
double dot(const double *a, const double *b) {
  double s = 0;
  for (int i = 0; i < 3; ++i)
    s += a[i] * b[i];
  return s;
}
inline double p2(double x) { return x * x; }

// ---------------------------------------------------------------------------
// equations of state (EOSX)
// ---------------------------------------------------------------------------
struct Range {
  double min, max;
};

struct Ideal { // eos_3p_idealgas.hxx:115-229
  double gamma, gm1, inv_gamma, temp_over_eps;
  Range rgrho, rgye, rgtemp, rgeps;
  double press_re(double rho, double &eps, double) const { return gm1 * rho * eps; }
  double eps_rp(double rho, double press, double) const { return press / (rho * gm1); }
  double csnd_re(double, double &eps, double) const {
    return std::sqrt(gm1 * eps / (eps + inv_gamma));
  }
  double temp_re(double, double &eps, double) const { return temp_over_eps * eps; }
  double eps_rt(double, double temp, double) const { return temp / temp_over_eps; }
  double press_rt(double rho, double temp, double ye) const {
    double e = eps_rt(rho, temp, ye);
    return press_re(rho, e, ye);
  }
  double kappa_re(double rho, double &eps, double) const {
    return (gamma - 1.0) * eps * std::pow(rho, 1.0 - gamma);
  }
  double gamma_noble() const { return gamma; }
};

struct Poly { // eos_1p_polytropic.hxx:57-90
  double k, gamma, n, np1, invn, rho_p;
  double gm1_rho(double rho) const { return np1 * std::pow(rho / rho_p, invn); }
  double sed_gm1(double gm1) const { return gm1 / gamma; }
};

// Uniform trilinear table (eos_linear_interp_ND.hxx:30-231), 19 variables
// interleaved variable-fastest, axes ln(rho), ln(T), Ye.
struct Table {
  int n[3];
  std::vector<double> x[3];
  std::vector<double> y;
  double dx[3], idx[3];
  static constexpr int NV = 19;
  size_t find(int d, double xin) const {
    const double xL = xin - x[d][0];
    if (xL <= 0)
      return 0;
    const int index = static_cast<int>(xL * idx[d]);
    if ((size_t)index > (size_t)(n[d] - 2))
      return n[d] - 2;
    return index;
  }
  static double lin(double A, double B, double xA, double xB, double xv) {
    const double lam = (xv - xA) / (xB - xA);
    return (B - A) * lam + A;
  }
  double interp(int var, double a, double b, double c) const {
    const size_t i = find(0, a), j = find(1, b), k = find(2, c);
    double Bk[2];
    for (int o2 = 0; o2 < 2; ++o2) {
      double Aj[2];
      for (int o1 = 0; o1 < 2; ++o1) {
        const size_t base = i + n[0] * ((j + o1) + n[1] * (k + o2));
        Aj[o1] = lin(y[var + NV * base], y[var + NV * (base + 1)], x[0][i], x[0][i + 1], a);
      }
      Bk[o2] = lin(Aj[0], Aj[1], x[1][j], x[1][j + 1], b);
    }
    return lin(Bk[0], Bk[1], x[2][k], x[2][k + 1], c);
  }
};

// Brent's zero finder on a sign-change interval (eos_brent.hxx:7-170; R. P.
// Brent, "Algorithms for Minimization without Derivatives", ch. 4).
template <class Fn> double zero_brent(double a, double b, double t, Fn &&f) {
  double sa = a, sb = b, fa = f(sa), fb = f(sb);
  double c = sa, fc = fa, e = sb - sa, d = e;
  const double macheps = std::numeric_limits<double>::epsilon();
  for (int it = 0; it < 10000; ++it) {
    if (std::fabs(fc) < std::fabs(fb)) {
      sa = sb;
      sb = c;
      c = sa;
      fa = fb;
      fb = fc;
      fc = fa;
    }
    const double tol = 2.0 * macheps * std::fabs(sb) + t;
    const double m = 0.5 * (c - sb);
    if (std::fabs(m) <= tol || fb == 0.0)
      break;
    if (std::fabs(e) < tol || std::fabs(fa) <= std::fabs(fb)) {
      e = m;
      d = e;
    } else {
      double s = fb / fa, p, q;
      if (sa == c) {
        p = 2.0 * m * s;
        q = 1.0 - s;
      } else {
        q = fa / fc;
        const double r = fb / fc;
        p = s * (2.0 * m * q * (q - r) - (sb - sa) * (r - 1.0));
        q = (q - 1.0) * (r - 1.0) * (s - 1.0);
      }
      if (0.0 < p)
        q = -q;
      else
        p = -p;
      s = e;
      e = d;
      if (2.0 * p < 3.0 * m * q - std::fabs(tol * q) && p < std::fabs(0.5 * s * q)) {
        d = p / q;
      } else {
        e = m;
        d = e;
      }
    }
    sa = sb;
    fa = fb;
    if (tol < std::fabs(d))
      sb = sb + d;
    else if (0.0 < m)
      sb = sb + tol;
    else
      sb = sb - tol;
    fb = f(sb);
    if ((0.0 < fb && 0.0 < fc) || (fb <= 0.0 && fc <= 0.0)) {
      c = sa;
      fc = fa;
      e = sb - sa;
      d = e;
    }
  }
  return sb;
}

struct Tab { // eos_3p_tabulated3d.hxx:197-367
  enum { PRESS = 0, EPS = 1, S = 2, CS2 = 4 };
  Table t;
  double shift;
  Range rgrho, rgye, rgtemp, rgeps;
  double logtemp(double rho, double &eps, double ye) const {
    const double r = std::fmin(std::fmax(rho, rgrho.min), rgrho.max);
    eps = std::fmax(eps + shift, rgeps.min + shift) - shift;
    const double lrho = std::log(r);
    const double leps = std::log(eps + shift);
    const double x1min = t.x[1].front(), x1max = t.x[1].back();
    const double vmin = t.interp(EPS, lrho, x1min, ye);
    const double vmax = t.interp(EPS, lrho, x1max, ye);
    if (leps <= vmin) {
      eps = std::exp(vmin) - shift;
      return x1min;
    }
    if (leps >= vmax) {
      eps = std::exp(vmax) - shift;
      return x1max;
    }
    return zero_brent(x1min, x1max, 1.e-14,
                      [&](double lt) { return leps - t.interp(EPS, lrho, lt, ye); });
  }
  double lr_clamped(double rho) const {
    return std::log(std::fmin(std::fmax(rho, rgrho.min), rgrho.max));
  }
  double lt_clamped(double temp) const {
    return std::log(std::fmin(std::fmax(temp, rgtemp.min), rgtemp.max));
  }
  double press_re(double rho, double &eps, double ye) const {
    const double lr = lr_clamped(rho);
    const double lt = logtemp(rho, eps, ye);
    return std::exp(t.interp(PRESS, lr, lt, ye));
  }
  double press_rt(double rho, double temp, double ye) const {
    // takes the logs of the unclamped inputs, as the reference does (:234-236)
    return std::exp(t.interp(PRESS, std::log(rho), std::log(temp), ye));
  }
  double eps_rt(double rho, double temp, double ye) const {
    return std::exp(t.interp(EPS, lr_clamped(rho), lt_clamped(temp), ye)) - shift;
  }
  double eps_rp(double, double, double) const {
    throw Fail("tabulated EOS: eps(rho, press) is not available (reference asserts)");
  }
  double csnd_re(double rho, double &eps, double ye) const {
    const double lr = lr_clamped(rho);
    const double lt = logtemp(rho, eps, ye);
    return std::sqrt(t.interp(CS2, lr, lt, ye));
  }
  double temp_re(double rho, double &eps, double ye) const {
    return std::exp(logtemp(rho, eps, ye));
  }
  double entropy_rt(double rho, double temp, double ye) const {
    return t.interp(S, lr_clamped(rho), lt_clamped(temp), ye);
  }
  double kappa_re(double rho, double &eps, double ye) const {
    return entropy_rt(rho, temp_re(rho, eps, ye), ye);
  }
  double gamma_noble() const { return std::numeric_limits<double>::quiet_NaN(); }
};

Ideal g_ideal;
Tab g_tab;
Poly g_poly;
int g_eos_kind = -1; // 0 ideal, 1 tabulated

// ---------------------------------------------------------------------------
// reconstruction (ReconX)
// ---------------------------------------------------------------------------
int sgn(double v) { return (0.0 < v) - (v < 0.0); }
double minmod(double x, double y) { // minmod.hxx:13-25
  if (std::signbit(x) != std::signbit(y))
    return 0.0;
  return std::fabs(x) < std::fabs(y) ? x : y;
}
double monocentral(double x, double y) { // monocentral.hxx:15-26
  if (sgn(x) != sgn(y))
    return 0;
  return sgn(x) * std::min(2 * std::fabs(x), std::min(2 * std::fabs(y), std::fabs(x + y) / 2));
}

// ppm.hxx:21-161 for cell I with neighbours Imm..Ipp; returns {low, up}
void ppm_cell(double gImm, double gIm, double gI, double gIp, double gIpp,
              double pImm, double pIm, double pIp, double pIpp, double vIm,
              double vIp, bool is_rho, double out[2]) {
  const axb_params &P = g_p;
  const double diff_Im = gI - gImm, diff_I = gIp - gIm, diff_Ip = gIpp - gI;
  const double d_Im = 0.5 * diff_Im, d_I = 0.5 * diff_I, d_Ip = 0.5 * diff_Ip;
  const double a1 = 2 * std::fabs(gIm - gImm), a2 = 2 * std::fabs(gI - gIm),
               a3 = 2 * std::fabs(gIp - gI), a4 = 2 * std::fabs(gIpp - gIp);
  const bool s1 = (gI - gIm) * (gIm - gImm) > 0;
  const bool s2 = (gIp - gI) * (gI - gIm) > 0;
  const bool s3 = (gIpp - gIp) * (gIp - gI) > 0;
  const double m1 = s1 ? sgn(d_Im) * std::min(std::fabs(d_Im), std::min(a1, a2)) : 0;
  const double m2 = s2 ? sgn(d_I) * std::min(std::fabs(d_I), std::min(a2, a3)) : 0;
  const double m3 = s3 ? sgn(d_Ip) * std::min(std::fabs(d_Ip), std::min(a3, a4)) : 0;
  double lo = 0.5 * (gIm + gI) + (1. / 6.) * (m1 - m2);
  double up = 0.5 * (gI + gIp) + (1. / 6.) * (m2 - m3);
  const double dp = pIp - pIm;
  const double minp = std::min(pIm, pIp);
  if (P.ppm_shock_detection && is_rho) {
    const double kg = P.poly_k * P.poly_gamma;
    if (kg * std::fabs(diff_I) * minp >= std::fabs(dp) * std::min(gIp, gIm)) {
      const double d2m = gI - 2 * gIm + gImm;
      const double d2p = gIpp - 2 * gIp + gI;
      const bool c2 = (std::fabs(diff_I) - P.ppm_eps_shock * std::min(std::fabs(gIp), std::fabs(gIm))) > 0.;
      const double et = ((d2m * d2p < 0) && c2) ? ((-1. / 6.) * (d2p - d2m) / diff_I) : 0;
      const double eta = std::max(0., std::min(P.ppm_eta1 * (et - P.ppm_eta2), 1.));
      lo = (1 - eta) * lo + eta * (gIm + 0.5 * m1);
      up = (1 - eta) * up + eta * (gIp - 0.5 * m3);
    }
  }
  if (P.ppm_zone_flattening) {
    const double w = ((std::fabs(dp) > P.ppm_eps * minp) && (vIm > vIp)) ? 1. : 0;
    const double ft = (std::fabs(pIpp - pImm) < P.ppm_small)
                          ? 1.0
                          : std::max(0., 1. - w * std::max(0., P.ppm_omega2 *
                                                                   ((dp / (pIpp - pImm)) -
                                                                    P.ppm_omega1)));
    const double r = (1 - ft) * gI;
    lo = ft * lo + r;
    up = ft * up + r;
  }
  if ((up - gI) * (gI - lo) <= 0) {
    lo = gI;
    up = gI;
  } else {
    const double dr = up - lo;
    const double dr2 = dr * dr;
    const double g6 = 6 * dr * (gI - 0.5 * (lo + up));
    if (g6 > dr2)
      lo = 3 * gI - 2 * up;
    else if (g6 < -dr2)
      up = 3 * gI - 2 * lo;
  }
  out[0] = lo;
  out[1] = up;
}

// wenoz.hxx:21-102 for cell I; returns {minus (low), plus (up)}
void wenoz_cell(double a, double b, double c, double d, double e, double weps,
                double out[2]) {
  const double be[3] = {(13.0 / 12.0) * p2(a - 2.0 * b + c) + (1.0 / 4.0) * p2(a - 4.0 * b + 3.0 * c),
                        (13.0 / 12.0) * p2(b - 2.0 * c + d) + (1.0 / 4.0) * p2(b - d),
                        (13.0 / 12.0) * p2(c - 2.0 * d + e) + (1.0 / 4.0) * p2(3.0 * c - 4.0 * d + e)};
  const double t5 = std::fabs(be[0] - be[2]);
  double ax[3];
  for (int q = 0; q < 3; ++q)
    ax[q] = 1.0 + t5 / (be[q] + weps);
  const double wt[3] = {3.0 / 10.0, 3.0 / 5.0, 1.0 / 10.0};
  const double am[3] = {wt[0] * ax[0], wt[1] * ax[1], wt[2] * ax[2]};
  const double ap[3] = {wt[2] * ax[0], wt[1] * ax[1], wt[0] * ax[2]};
  const double dm = am[0] + am[1] + am[2], dpp = ap[0] + ap[1] + ap[2];
  const double om[3] = {am[0] / dm, am[1] / dm, am[2] / dm};
  const double op[3] = {ap[0] / dpp, ap[1] / dpp, ap[2] / dpp};
  out[0] = (om[2] / 6.0) * (2.0 * e - 7.0 * d + 11.0 * c) +
           (om[1] / 6.0) * (-1.0 * d + 5.0 * c + 2.0 * b) +
           (om[0] / 6.0) * (2.0 * c + 5.0 * b - 1.0 * a);
  out[1] = (op[0] / 6.0) * (2.0 * a - 7.0 * b + 11.0 * c) +
           (op[1] / 6.0) * (-1.0 * b + 5.0 * c + 2.0 * d) +
           (op[2] / 6.0) * (2.0 * c + 5.0 * d - 1.0 * e);
}

// mp5.hxx:24-77, value of the middle cell on the side of the 4th argument
double mp5(double Imm, double Im, double I, double Ip, double Ipp, double al) {
  const double ul = (2 * Imm - 13 * Im + 47 * I + 27 * Ip - 3 * Ipp) / 60.0;
  const double dmn = I - Im, dpl = Ip - I;
  const double ump = I + minmod(dpl, al * dmn);
  if ((ul - I) * (ul - ump) <= 1.0e-10)
    return ul;
  const double dm = Imm + I - 2 * Im, dd = Im + Ip - 2 * I, dp = I + Ipp - 2 * Ip;
  const double dmp = minmod(minmod(4 * dd - dp, 4 * dp - dd), minmod(dd, dp));
  const double dmm = minmod(minmod(4 * dm - dd, 4 * dd - dm), minmod(dm, dd));
  const double uul = I + al * dmn, uav = (I + Ip) / 2.0, umd = uav - dmp / 2.0;
  const double ulc = I + dmn / 2.0 + 4.0 / 3.0 * dmm;
  const double umin = std::max(std::min(I, std::min(Ip, umd)), std::min(I, std::min(uul, ulc)));
  const double umax = std::min(std::max(I, std::max(Ip, umd)), std::max(I, std::max(uul, ulc)));
  return ul + minmod(umin - ul, umax - ul);
}

// ReconX::reconstruct (reconstruct.hxx:36-103) on v[0..5] = Immm..Ippp.
void recon_face(int method, const double *v, const double *pr, const double *vel,
                bool is_rho, double out[2]) {
  switch (method) {
  case AXB_RECON_GODUNOV:
    out[0] = v[2];
    out[1] = v[3];
    return;
  case AXB_RECON_MINMOD:
    out[0] = v[2] + minmod(v[3] - v[2], v[2] - v[1]) / 2;
    out[1] = v[3] - minmod(v[4] - v[3], v[3] - v[2]) / 2;
    return;
  case AXB_RECON_MONOCENTRAL:
    out[0] = v[2] + monocentral(v[3] - v[2], v[2] - v[1]) / 2;
    out[1] = v[3] - monocentral(v[4] - v[3], v[3] - v[2]) / 2;
    return;
  case AXB_RECON_PPM: {
    double a[2], b[2];
    ppm_cell(v[0], v[1], v[2], v[3], v[4], pr[0], pr[1], pr[3], pr[4], vel[1], vel[3], is_rho, a);
    ppm_cell(v[1], v[2], v[3], v[4], v[5], pr[1], pr[2], pr[4], pr[5], vel[2], vel[4], is_rho, b);
    out[0] = a[1];
    out[1] = b[0];
    return;
  }
  case AXB_RECON_WENOZ: {
    double a[2], b[2];
    wenoz_cell(v[0], v[1], v[2], v[3], v[4], g_p.weno_eps, a);
    wenoz_cell(v[1], v[2], v[3], v[4], v[5], g_p.weno_eps, b);
    out[0] = a[1];
    out[1] = b[0];
    return;
  }
  case AXB_RECON_MP5:
    out[0] = mp5(v[0], v[1], v[2], v[3], v[4], g_p.mp5_alpha);
    out[1] = mp5(v[5], v[4], v[3], v[2], v[1], g_p.mp5_alpha);
    return;
  }
  throw Fail("reconstruction method not restated (eppm)");
}

// ---------------------------------------------------------------------------
// face physics (fluxes.cxx:216-795, eigenvalues.hxx:19-79, fluxes.hxx:20-49)
// ---------------------------------------------------------------------------
template <class EOS>
void calc_flux(const EOS &eos, int dir) {
  const int d1 = (dir + 1) % 3, d2 = (dir + 2) % 3;
  const char *names[3][10] = {
      {"fxdens", "fxmomx", "fxmomy", "fxmomz", "fxtau", "fxDYe", "fxDEnt", "fxBx", "fxBy", "fxBz"},
      {"fydens", "fymomx", "fymomy", "fymomz", "fytau", "fyDYe", "fyDEnt", "fyBx", "fyBy", "fyBz"},
      {"fzdens", "fzmomx", "fzmomy", "fzmomz", "fztau", "fzDYe", "fzDEnt", "fzBx", "fzBy", "fzBz"}};
  double *out[10];
  for (int q = 0; q < 10; ++q)
    out[q] = F(names[dir][q]);
  const char *bnames[3][2] = {{"fxBy", "fxBz"}, {"fyBx", "fyBz"}, {"fzBx", "fzBy"}};
  const double *rho = need("rho"), *ent = need("entropy"), *ye = need("Ye"),
               *press = need("press");
  const bool with_temp = g_p.reconstruct_with_temperature != 0;
  const double *temp = with_temp ? need("temperature") : nullptr;
  const double *vel[3] = {need("velx"), need("vely"), need("velz")};
  const double *Bv[3] = {need("Bvecx"), need("Bvecy"), need("Bvecz")};
  const double *dBs[3] = {need("dBx_stag"), need("dBy_stag"), need("dBz_stag")};
  const double *alp = need("alp");
  const double *beta[3] = {need("betax"), need("betay"), need("betaz")};
  const double *g[6] = {need("gxx"), need("gxy"), need("gxz"), need("gyy"), need("gyz"), need("gzz")};
  const long long s = st(dir), s1 = st(d1), s2 = st(d2);
  const int cen[3] = {dir != 0, dir != 1, dir != 2};
  loop(cen[0], cen[1], cen[2], [&](int i, int j, int k) {
    const long long I = at(i, j, k);
    auto v2f = [&](const double *f) {
      double a = 0.0;
      for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
          a += f[I + s1 * dj + s2 * dk];
      return a / 4.0;
    };
    const double alp_avg = v2f(alp);
    double bavg[3];
    for (int q = 0; q < 3; ++q)
      bavg[q] = v2f(beta[q]);
    const Sym G{v2f(g[0]), v2f(g[1]), v2f(g[2]), v2f(g[3]), v2f(g[4]), v2f(g[5])};
    const double detg = det(G), sqrtg = std::sqrt(detg);
    auto rec = [&](const double *f, int method, bool is_rho, double o[2]) {
      double v[6], pr[6], vd[6];
      for (int m = 0; m < 6; ++m) {
        v[m] = f[I + (m - 3) * s];
        pr[m] = press[I + (m - 3) * s];
        vd[m] = vel[dir][I + (m - 3) * s];
      }
      recon_face(method, v, pr, vd, is_rho, o);
    };
    const int hi = g_p.reconstruction_method, lo = g_p.loworder_method;
    // the thermodynamic variable reconstructed beside rho, entropy and Ye:
    // the temperature or the pressure (fluxes.cxx:257-355)
    const double *thermo = with_temp ? temp : press;
    double r_rho[2], r_ent[2], r_ye[2], r_p[2], r_t[2];
    rec(rho, hi, true, r_rho);
    rec(ent, hi, false, r_ent);
    rec(ye, hi, false, r_ye);
    rec(thermo, hi, false, r_t);
    const bool lo0 = r_rho[0] <= 0.0 || r_ent[0] <= 0.0 || r_ye[0] <= 0.0 || r_t[0] <= 0.0;
    const bool lo1 = r_rho[1] <= 0.0 || r_ent[1] <= 0.0 || r_ye[1] <= 0.0 || r_t[1] <= 0.0;
    auto lowfix = [&](const double *f, bool is_rho, double o[2]) {
      double t[2];
      if (lo0) {
        rec(f, lo, is_rho, t);
        o[0] = t[0];
      }
      if (lo1) {
        rec(f, lo, is_rho, t);
        o[1] = t[1];
      }
    };
    lowfix(rho, true, r_rho);
    lowfix(ent, false, r_ent);
    lowfix(ye, false, r_ye);
    lowfix(thermo, false, r_t);
    double eps[2];
    for (int f = 0; f < 2; ++f) {
      if (with_temp) {
        eps[f] = eos.eps_rt(r_rho[f], r_t[f], r_ye[f]);
        r_p[f] = eos.press_rt(r_rho[f], r_t[f], r_ye[f]);
      } else {
        r_p[f] = r_t[f];
        eps[f] = eos.eps_rp(r_rho[f], r_p[f], r_ye[f]);
        (void)eos.temp_re(r_rho[f], eps[f], r_ye[f]); // may clamp eps (tabulated)
      }
    }
    double B[3][2];
    B[dir][0] = B[dir][1] = dBs[dir][I] / sqrtg;
    for (int q : {d1, d2}) {
      rec(Bv[q], hi, false, B[q]);
      lowfix(Bv[q], false, B[q]);
    }
    double V[3][2];
    for (int q = 0; q < 3; ++q) {
      rec(vel[q], hi, false, V[q]);
      lowfix(vel[q], false, V[q]);
    }
    double U[10][2], Fl[10][2], lam[2][2];
    for (int f = 0; f < 2; ++f) {
      const double v[3] = {V[0][f], V[1][f], V[2][f]};
      const double b[3] = {B[0][f], B[1][f], B[2][f]};
      double vl[3], Bl[3];
      mul(G, v, vl);
      const double W = 1 / std::sqrt(1 - dot(vl, v));
      double vt[3];
      for (int q = 0; q < 3; ++q)
        vt[q] = alp_avg * v[q] - bavg[q];
      const double ab0 = W * dot(b, vl);
      mul(G, b, Bl);
      const double B2 = dot(b, Bl);
      double bl[3];
      for (int q = 0; q < 3; ++q)
        bl[q] = Bl[q] / W + ab0 * vl[q];
      const double bsq = (B2 + p2(ab0)) / p2(W);
      double e = eps[f];
      const double cs = eos.csnd_re(r_rho[f], e, r_ye[f]);
      const double cs2 = cs * eos.csnd_re(r_rho[f], e, r_ye[f]);
      const double h = 1 + e + r_p[f] / r_rho[f];
      const double dens = sqrtg * r_rho[f] * W;
      const double DEnt = sqrtg * r_rho[f] * W * r_ent[f];
      const double dhW = dens * h * W;
      const double dhWp = dhW + sqrtg * (p2(ab0) + B2);
      const double ppm = r_p[f] + 0.5 * bsq;
      const double vtd = vt[dir];
      const double as = alp_avg * sqrtg;
      const double BoW = b[dir] / W;
      U[0][f] = dens;
      Fl[0][f] = dens * vtd;
      for (int q = 0; q < 3; ++q) {
        const double mom = dhWp * vl[q] - sqrtg * ab0 * bl[q];
        U[1 + q][f] = mom;
        Fl[1 + q][f] = mom * vtd + as * (ppm * (q == dir ? 1.0 : 0.0) - bl[q] * BoW);
      }
      const double tau = dhW - dens + sqrtg * (B2 - ppm);
      U[4][f] = tau;
      Fl[4][f] = tau * vtd + as * (ppm * v[dir] - ab0 * BoW);
      U[5][f] = dens * r_ye[f];
      Fl[5][f] = U[5][f] * vtd;
      U[6][f] = DEnt;
      Fl[6][f] = DEnt * vtd;
      double Bt[3];
      for (int q = 0; q < 3; ++q)
        Bt[q] = sqrtg * b[q];
      double E[3];
      for (int q = 0; q < 3; ++q) {
        const int a1 = (q + 1) % 3, a2 = (q + 2) % 3;
        E[q] = Bt[a1] * vt[a2] - Bt[a2] * vt[a1];
      }
      for (int q = 0; q < 3; ++q) {
        const int a1 = (q + 1) % 3, a2 = (q + 2) % 3;
        const double u1 = a1 == dir ? 1.0 : 0.0, u2 = a2 == dir ? 1.0 : 0.0;
        U[7 + q][f] = Bt[q];
        Fl[7 + q][f] = u1 * E[a2] - u2 * E[a1];
      }
      const double be = bavg[dir];
      const double uinv = inv(G, detg)(dir, dir);
      const double a0 = (bsq + cs2 * h * r_rho[f]) * (p2(be) - p2(alp_avg) * uinv) -
                        (-1 + cs2) * h * r_rho[f] * p2(be - alp_avg * v[dir]) * p2(W);
      const double a1 = 2 * be * (bsq + cs2 * h * r_rho[f]) -
                        2 * (-1 + cs2) * h * r_rho[f] * (be - alp_avg * v[dir]) * p2(W);
      const double a2 = bsq + h * r_rho[f] * (cs2 + p2(W) - cs2 * p2(W));
      double dt = p2(a1) - 4 * a2 * a0;
      if (dt < 0)
        dt = 0;
      lam[f][0] = ((-a1 + std::sqrt(dt)) / (2 * a2)) / alp_avg;
      lam[f][1] = ((-a1 - std::sqrt(dt)) / (2 * a2)) / alp_avg;
    }
    const double l8[8] = {lam[0][0], lam[0][0], lam[0][1], lam[0][1],
                          lam[1][0], lam[1][0], lam[1][1], lam[1][1]};
    for (int q = 0; q < 10; ++q) {
      double r = ora_riemann(g_p.flux_type, l8, U[q][0], U[q][1], Fl[q][0], Fl[q][1]);
      if (q >= 7)
        r = (q - 7 != dir) * r;
      if (out[q])
        out[q][I] = r;
    }
    (void)bnames;
  });
}

// ---------------------------------------------------------------------------
// CalcAuxForAvecPsi (fluxes.cxx:798-826)
// ---------------------------------------------------------------------------
void calc_aux() {
  const double *A[3] = {need("Avec_x"), need("Avec_y"), need("Avec_z")};
  const double *g[6] = {need("gxx"), need("gxy"), need("gxz"), need("gyy"), need("gyz"), need("gzz")};
  const double *beta[3] = {need("betax"), need("betay"), need("betaz")};
  const double *alp = need("alp"), *Psi = need("Psi");
  double *o[7] = {need("Fx"), need("Fy"), need("Fz"), need("Fbetax"), need("Fbetay"), need("Fbetaz"), need("G")};
  loop(0, 0, 0, [&](int i, int j, int k) {
    const long long I = at(i, j, k);
    double Av[3];
    for (int d = 0; d < 3; ++d) {
      double s = 0.0;
      for (int di = 0; di < 2; ++di)
        s += A[d][I - st(d) * di];
      Av[d] = s / 2.0;
    }
    const Sym G{g[0][I], g[1][I], g[2][I], g[3][I], g[4][I], g[5][I]};
    const double be[3] = {beta[0][I], beta[1][I], beta[2][I]};
    const double dg = det(G), sg = std::sqrt(dg);
    const Sym ug = inv(G, dg);
    double Aup[3];
    mul(ug, Av, Aup);
    for (int q = 0; q < 3; ++q) {
      o[q][I] = alp[I] * sg * Aup[q];
      o[3 + q][I] = be[q] * Psi[I];
    }
    o[6][I] = alp[I] * Psi[I] / sg - dot(be, Av);
  });
}

// ---------------------------------------------------------------------------
// SourceTerms<FDORDER> (source.cxx:20-168), calc_fd_v2c (aster_fd.hxx:49-110)
// ---------------------------------------------------------------------------
double fd_v2c(int order, const double *f, long long I, int d) {
  const int a = (d + 1) % 3, b = (d + 2) % 3;
  const long long s = st(d);
  const long long base[4] = {I, I + st(a), I + st(b), I + st(a) + st(b)};
  double e[4];
  for (int q = 0; q < 4; ++q) {
    const long long J = base[q];
    if (order == 2)
      e[q] = (f[J + s] - f[J]) / g_box.dx[d];
    else
      e[q] = ((1.0 / 24.0) * f[J - s] - (27.0 / 24.0) * f[J] + (27.0 / 24.0) * f[J + s] -
              (1.0 / 24.0) * f[J + 2 * s]) /
             g_box.dx[d];
  }
  return 0.25 * (e[0] + e[1] + e[2] + e[3]);
}

void source_terms() {
  const int fd = g_p.local_spatial_order;
  if (fd != 2 && fd != 4)
    throw Fail("local_spatial_order must be set to 2 or 4.");
  const double *alp = need("alp");
  const double *beta[3] = {need("betax"), need("betay"), need("betaz")};
  const double *g[6] = {need("gxx"), need("gxy"), need("gxz"), need("gyy"), need("gyz"), need("gzz")};
  const double *K[6] = {need("kxx"), need("kxy"), need("kxz"), need("kyy"), need("kyz"), need("kzz")};
  const double *vel[3] = {need("velx"), need("vely"), need("velz")};
  const double *Bv[3] = {need("Bvecx"), need("Bvecy"), need("Bvecz")};
  const double *rho = need("rho"), *eps = need("eps"), *press = need("press");
  double *r[7] = {need("densrhs"), need("momxrhs"), need("momyrhs"), need("momzrhs"),
                  need("taurhs"), need("DYe_rhs"), need("DEntrhs")};
  loop(1, 1, 1, [&](int i, int j, int k) {
    const long long I = at(i, j, k);
    auto v2c = [&](const double *f) {
      double s = 0.0;
      for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
          for (int di = 0; di < 2; ++di)
            s += f[I + di + g_box.sy * dj + g_box.sz * dk];
      return s / 8.0;
    };
    const double a = v2c(alp);
    double b[3];
    for (int q = 0; q < 3; ++q)
      b[q] = v2c(beta[q]);
    const Sym G{v2c(g[0]), v2c(g[1]), v2c(g[2]), v2c(g[3]), v2c(g[4]), v2c(g[5])};
    const Sym Kc{v2c(K[0]), v2c(K[1]), v2c(K[2]), v2c(K[3]), v2c(K[4]), v2c(K[5])};
    const double dg = det(G), sdg = std::sqrt(dg);
    const Sym ug = inv(G, dg);
    double da[3], db[3][3];
    Sym dG[3];
    for (int d = 0; d < 3; ++d) {
      da[d] = fd_v2c(fd, alp, I, d);
      for (int q = 0; q < 3; ++q)
        db[d][q] = fd_v2c(fd, beta[q], I, d);
      dG[d] = Sym{fd_v2c(fd, g[0], I, d), fd_v2c(fd, g[1], I, d), fd_v2c(fd, g[2], I, d),
                  fd_v2c(fd, g[3], I, d), fd_v2c(fd, g[4], I, d), fd_v2c(fd, g[5], I, d)};
    }
    const double vu[3] = {vel[0][I], vel[1][I], vel[2][I]};
    double vl[3];
    mul(G, vu, vl);
    const double w = 1.0 / std::sqrt(1.0 - dot(vl, vu));
    const double rhW2 = (rho[I] * (1.0 + eps[I]) + press[I]) * w * w;
    double vs[3];
    for (int q = 0; q < 3; ++q)
      vs[q] = vu[q] - b[q] / a;
    const double Bu[3] = {Bv[0][I], Bv[1][I], Bv[2][I]};
    double Bl[3];
    mul(G, Bu, Bl);
    const double bs0 = w * dot(Bu, vl) / a;
    double bs[3];
    for (int q = 0; q < 3; ++q)
      bs[q] = Bu[q] / w + a * bs0 * vs[q];
    const double bs2 = (dot(Bu, Bl) + p2(a * bs0)) / p2(w);
    double gb[3], gbs[3], bsl[3];
    mul(G, b, gb);
    mul(G, bs, gbs);
    for (int q = 0; q < 3; ++q)
      bsl[q] = gb[q] * bs0 + gbs[q];
    const double A = rhW2 + bs2 * p2(w);
    const double P = press[I] + 0.5 * bs2;
    const double t00 = (A - P) / p2(a) - p2(bs0);
    double t0[3], t0l[3];
    for (int q = 0; q < 3; ++q) {
      t0[q] = A * vs[q] / a + P * b[q] / p2(a) - bs0 * bs[q];
      t0l[q] = A * vl[q] / a - bsl[q] * bs0;
    }
    // T^{ij} is a symmetric matrix: built from its upper triangle and
    // mirrored, as the smat it is in the reference
    double t[3][3];
    for (int p = 0; p < 3; ++p)
      for (int q = p; q < 3; ++q)
        t[p][q] = t[q][p] =
            A * vs[p] * vs[q] + P * (ug(p, q) - b[p] * b[q] / p2(a)) - bs[p] * bs[q];
    double sk[3];
    mul(Kc, b, sk);
    const double ssk = dot(sk, b);
    double X[3];
    for (int q = 0; q < 3; ++q)
      X[q] = -da[q] + 2.0 * sk[q];
    double Kt = 0;
    for (int p = 0; p < 3; ++p)
      for (int q = 0; q < 3; ++q)
        Kt += Kc(p, q) * t[p][q];
    const double taus = t00 * (ssk - dot(b, da)) + dot(t0, X) + Kt;
    double ms[3];
    for (int d = 0; d < 3; ++d) {
      double nrm = 0, c1 = 0, c3 = 0;
      for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) {
          nrm += dG[d](p, q) * b[p] * b[q];
          c1 += dG[d](p, q) * t0[p] * b[q];
          c3 += t[p][q] * dG[d](p, q);
        }
      ms[d] = t00 * (0.5 * nrm - a * da[d]) + c1 + dot(t0l, db[d]) + 0.5 * c3;
    }
    r[0][I] = 0.0;
    r[6][I] = 0.0;
    r[1][I] = a * sdg * ms[0];
    r[2][I] = a * sdg * ms[1];
    r[3][I] = a * sdg * ms[2];
    r[4][I] = a * sdg * taus;
    r[5][I] = 0.0;
  });
}

// ---------------------------------------------------------------------------
// AsterX_RHS (rhs.cxx:107-252): flux divergence, flux-CT E, gauge
// ---------------------------------------------------------------------------
void rhs() {
  const char *fn[7][3] = {{"fxdens", "fydens", "fzdens"}, {"fxmomx", "fymomx", "fzmomx"},
                          {"fxmomy", "fymomy", "fzmomy"}, {"fxmomz", "fymomz", "fzmomz"},
                          {"fxtau", "fytau", "fztau"},    {"fxDYe", "fyDYe", "fzDYe"},
                          {"fxDEnt", "fyDEnt", "fzDEnt"}};
  double *r[7] = {need("densrhs"), need("momxrhs"), need("momyrhs"), need("momzrhs"),
                  need("taurhs"), need("DYe_rhs"), need("DEntrhs")};
  const double idx[3] = {1 / g_box.dx[0], 1 / g_box.dx[1], 1 / g_box.dx[2]};
  loop(1, 1, 1, [&](int i, int j, int k) {
    const long long I = at(i, j, k);
    for (int v = 0; v < 7; ++v) {
      double df[3];
      for (int d = 0; d < 3; ++d) {
        const double *f = need(fn[v][d]);
        df[d] = f[I + st(d)] - f[I];
      }
      r[v][I] += -dot(idx, df);
    }
  });
  // fBs(a)(b): flux along b of B_a
  const char *fB[3][3] = {{"fxBx", "fyBx", "fzBx"}, {"fxBy", "fyBy", "fzBy"}, {"fxBz", "fyBz", "fzBz"}};
  const double *G = need("G");
  const bool gl = g_p.vector_potential_gauge == AXB_GAUGE_GEN_LORENZ;
  const char *an[3] = {"Avec_x_rhs", "Avec_y_rhs", "Avec_z_rhs"};
  for (int e = 0; e < 3; ++e) {
    double *o = need(an[e]);
    const int ja = (e + 1) % 3, ka = (e + 2) % 3;
    const double *fjk = need(fB[ja][ka]), *fkj = need(fB[ka][ja]);
    loop(e == 0, e == 1, e == 2, [&](int i, int j, int k) {
      const long long I = at(i, j, k);
      const double E = 0.25 * ((fjk[I] + fjk[I - st(ja)]) - (fkj[I] + fkj[I - st(ka)]));
      o[I] = gl ? -E - (G[I + st(e)] - G[I]) / g_box.dx[e] : -E;
    });
  }
  double *pr = need("Psi_rhs");
  const double *Fv[3] = {need("Fx"), need("Fy"), need("Fz")};
  const double *Fb[3] = {need("Fbetax"), need("Fbetay"), need("Fbetaz")};
  const double *beta[3] = {need("betax"), need("betay"), need("betaz")};
  const double *alp = need("alp"), *Psi = need("Psi");
  loop(0, 0, 0, [&](int i, int j, int k) {
    const long long I = at(i, j, k);
    if (!gl) {
      pr[I] = 0.0;
      return;
    }
    double dF = 0.0;
    for (int d = 0; d < 3; ++d) {
      const long long s = st(d);
      const double c2c = (0.5 / g_box.dx[d]) * (Fv[d][I + s] - Fv[d][I - s]);
      const int sg = beta[d][I] < 0 ? -1 : 1;
      const double one = -sg * (Fb[d][I + 2 * sg * s] - 4.0 * Fb[d][I + sg * s] + 3.0 * Fb[d][I]) *
                         (0.5 / g_box.dx[d]);
      dF += c2c - one;
    }
    pr[I] = -dF - g_p.lorenz_damp_fac * alp[I] * Psi[I];
  });
}

// ---------------------------------------------------------------------------
// computeBfromA.cxx:20-85
// ---------------------------------------------------------------------------
void bstag() {
  const double *Ax = need("Avec_x"), *Ay = need("Avec_y"), *Az = need("Avec_z");
  double *b[3] = {need("dBx_stag"), need("dBy_stag"), need("dBz_stag")};
  const double idx[3] = {1 / g_box.dx[0], 1 / g_box.dx[1], 1 / g_box.dx[2]};
  for (int d = 0; d < 3; ++d)
    loop(d != 0, d != 1, d != 2, [&](int i, int j, int k) {
      const long long I = at(i, j, k), ip = I + 1, jp = I + g_box.sy, kp = I + g_box.sz;
      if (d == 0)
        b[0][I] = idx[1] * (Az[jp] - Az[I]) - idx[2] * (Ay[kp] - Ay[I]);
      else if (d == 1)
        b[1][I] = idx[2] * (Ax[kp] - Ax[I]) - idx[0] * (Az[ip] - Az[I]);
      else
        b[2][I] = idx[0] * (Ay[ip] - Ay[I]) - idx[1] * (Ax[jp] - Ax[I]);
    });
}

void dB_from_stag() {
  const double *s[3] = {need("dBx_stag"), need("dBy_stag"), need("dBz_stag")};
  double *o[3] = {need("dBx"), need("dBy"), need("dBz")};
  loop(1, 1, 1, [&](int i, int j, int k) {
    const long long I = at(i, j, k);
    for (int d = 0; d < 3; ++d)
      o[d][I] = 0.5 * (s[d][I] + s[d][I + st(d)]);
  });
}

// ---------------------------------------------------------------------------
// Con2PrimFactory (c2p.hxx, c2p_2DNoble.hxx, c2p_1DPalenzuela.hxx, cons.hxx,
// atmo.hxx) and the driver (con2prim.cxx:73-454)
// ---------------------------------------------------------------------------
struct Prim {
  double rho, eps, Ye, press, temp, ent, v[3], W, B[3], E[3];
  void nan() {
    const double n = std::numeric_limits<double>::quiet_NaN();
    rho = eps = Ye = press = temp = ent = W = n;
    for (int i = 0; i < 3; ++i)
      v[i] = B[i] = E[i] = n;
  }
};
struct Cons {
  double D, S[3], tau, DYe, DEnt, B[3];
  void nan() {
    const double n = std::numeric_limits<double>::quiet_NaN();
    D = tau = DYe = DEnt = n;
    for (int i = 0; i < 3; ++i)
      S[i] = B[i] = n;
  }
  void div(double s) {
    D /= s;
    tau /= s;
    for (int i = 0; i < 3; ++i)
      S[i] /= s;
    for (int i = 0; i < 3; ++i)
      B[i] /= s;
    DYe /= s;
    DEnt /= s;
  }
  void mul(double s) {
    D *= s;
    tau *= s;
    for (int i = 0; i < 3; ++i)
      S[i] *= s;
    for (int i = 0; i < 3; ++i)
      B[i] *= s;
    DYe *= s;
    DEnt *= s;
  }
};
struct Rep {
  int status = 13; // ERR_CODE_NOT_SET
  bool adjust = false, atmo = false;
  int iters = 0;
  bool failed() const { return status != 0; }
  void fail(int s) {
    status = s;
    atmo = false;
    adjust = true;
  }
};
struct Atmo {
  double rho, eps, ye, press, temp, ent, cut;
  void set(Prim &p) const {
    p.rho = rho;
    p.eps = eps;
    p.Ye = ye;
    p.press = press;
    p.temp = temp;
    p.ent = ent;
    for (int i = 0; i < 3; ++i)
      p.v[i] = 0.0, p.E[i] = 0.0;
    p.W = 1.0;
  }
  void set(Prim &p, Cons &c, const Sym &g) const {
    set(p);
    const double sd = std::sqrt(det(g));
    c.D = sd * rho;
    c.S[0] = c.S[1] = c.S[2] = 0.0;
    c.DYe = c.D * ye;
    c.DEnt = c.D * ent;
    double Bl[3];
    ::mul(g, p.B, Bl);
    c.tau = c.D * eps + 0.5 * sd * dot(p.B, Bl);
  }
};

void from_prim(Cons &c, const Prim &p, const Sym &g) { // cons.hxx:48-91
  const double sd = std::sqrt(det(g));
  double vl[3], Bl[3];
  ::mul(g, p.v, vl);
  const double W = p.W;
  ::mul(g, p.B, Bl);
  const double bst = W * dot(p.B, vl);
  double bl[3];
  for (int i = 0; i < 3; ++i)
    bl[i] = Bl[i] / W + bst * vl[i];
  const double bs2 = (dot(p.B, Bl) + bst * bst) / (W * W);
  c.D = sd * p.rho * W;
  const double h = W * W * (p.rho * (1.0 + p.eps) + p.press + bs2);
  for (int i = 0; i < 3; ++i)
    c.S[i] = sd * (h * vl[i] - bst * bl[i]);
  c.tau = sd * (h - (p.press + 0.5 * bs2) - bst * bst) - c.D;
  for (int i = 0; i < 3; ++i)
    c.B[i] = sd * p.B[i];
  c.DYe = c.D * p.Ye;
  c.DEnt = c.D * p.ent;
}

struct C2P {
  int maxit;
  double tol, cons_err, v_lim, w_lim, Bsq_lim, rho_BH, eps_BH, vwlim_BH;
  bool use_z, use_temp, use_press_atmo;
};
C2P c2p_params() {
  C2P c;
  c.maxit = g_p.max_iter;
  c.tol = g_p.c2p_tol;
  c.cons_err = g_p.cons_error_limit;
  c.w_lim = std::sqrt(1.0 + g_p.vw_lim * g_p.vw_lim);
  c.v_lim = g_p.vw_lim / c.w_lim;
  c.Bsq_lim = g_p.B_lim * g_p.B_lim;
  c.rho_BH = g_p.rho_BH;
  c.eps_BH = g_p.eps_BH;
  c.vwlim_BH = g_p.vwlim_BH;
  c.use_z = g_p.use_z;
  c.use_temp = g_p.use_temperature;
  c.use_press_atmo = g_p.use_press_atmo;
  return c;
}

void cons_floors(Cons &c, const Sym &g) { // c2p.hxx:330-369
  const double dg = det(g), sd = std::sqrt(dg);
  const Sym gu = inv(g, dg);
  double Bl[3];
  ::mul(g, c.B, Bl);
  const double tl = 0.5 * dot(Bl, c.B) / sd;
  if (c.tau <= tl)
    c.tau = tl;
  double Su[3];
  ::mul(gu, c.S, Su);
  const double S2 = dot(c.S, Su);
  const double sl = c.D + c.tau;
  if (S2 > sl * sl) {
    const double f = std::sqrt(sl * sl / S2);
    for (int i = 0; i < 3; ++i)
      c.S[i] = c.S[i] * f;
  }
}

template <class EOS>
void prim_floors(const EOS &eos, const C2P &cp, const Atmo &at_, Prim &p, const Cons &c,
                 const Sym &g, Rep &r) { // c2p.hxx:86-216
  bool re = false;
  if (p.Ye < eos.rgye.min) {
    p.Ye = eos.rgye.min;
    r.adjust = true;
    re = true;
  }
  if (p.Ye > eos.rgye.max) {
    p.Ye = eos.rgye.max;
    r.adjust = true;
    re = true;
  }
  double vl[3];
  ::mul(g, p.v, vl);
  const double sv = std::sqrt(dot(vl, p.v));
  auto keep_press = [&]() {
    re = false;
    p.eps = eos.eps_rp(p.rho, p.press, p.Ye);
    p.temp = eos.temp_re(p.rho, p.eps, p.Ye);
    p.ent = eos.kappa_re(p.rho, p.eps, p.Ye);
  };
  if (sv > cp.v_lim) {
    p.rho = c.D / cp.w_lim;
    const double f = cp.v_lim / sv;
    for (int i = 0; i < 3; ++i)
      p.v[i] *= f;
    p.W = cp.w_lim;
    r.adjust = true;
    if (cp.use_temp)
      re = true;
    else
      keep_press();
  }
  if (p.rho > eos.rgrho.max) {
    p.rho = eos.rgrho.max;
    r.adjust = true;
    if (cp.use_temp)
      re = true;
    else
      keep_press();
  }
  if (p.temp > eos.rgtemp.max) {
    p.temp = eos.rgtemp.max;
    re = true;
    r.adjust = true;
  }
  if (cp.use_press_atmo) {
    if (p.press < at_.press) {
      p.press = at_.press;
      p.eps = eos.eps_rp(p.rho, p.press, p.Ye);
      p.temp = eos.temp_re(p.rho, p.eps, p.Ye);
      p.ent = eos.kappa_re(p.rho, p.eps, p.Ye);
      re = false;
      r.adjust = true;
    }
  } else if (p.temp < at_.temp) {
    p.temp = at_.temp;
    re = true;
    r.adjust = true;
  }
  if (re) {
    p.eps = eos.eps_rt(p.rho, p.temp, p.Ye);
    p.press = eos.press_rt(p.rho, p.temp, p.Ye);
    p.ent = eos.kappa_re(p.rho, p.eps, p.Ye);
  }
}

void velocity(double Z, double W, double Bsq, double BiSi, bool use_z, Prim &p,
              const Cons &c, const Sym &gu, const Sym &gl) {
  if (use_z) {
    double z[3];
    for (int i = 0; i < 3; ++i) {
      z[i] = W * (gu(i, 0) * c.S[0] + gu(i, 1) * c.S[1] + gu(i, 2) * c.S[2]) / (Z + Bsq);
      z[i] += W * BiSi * c.B[i] / (Z * (Z + Bsq));
    }
    double zd[3];
    ::mul(gl, z, zd);
    const double L = std::sqrt(1.0 + (z[0] * zd[0] + z[1] * zd[1] + z[2] * zd[2]));
    for (int i = 0; i < 3; ++i)
      p.v[i] = z[i] / L;
    p.W = L;
  } else {
    for (int i = 0; i < 3; ++i) {
      p.v[i] = (gu(i, 0) * c.S[0] + gu(i, 1) * c.S[1] + gu(i, 2) * c.S[2]) / (Z + Bsq);
      p.v[i] += BiSi * c.B[i] / (Z * (Z + Bsq));
    }
    p.W = W;
  }
}
void efield(Prim &p, const Sym &gu) {
  double El[3];
  for (int i = 0; i < 3; ++i) {
    const int a = (i + 1) % 3, b = (i + 2) % 3;
    El[i] = p.B[a] * p.v[b] - p.B[b] * p.v[a];
  }
  ::mul(gu, El, p.E);
}

bool sylvester(const Sym &g, double dg) {
  return g.xx > 0.0 && g.xx * g.yy - g.xy * g.xy > 0.0 && dg > 0.0;
}

template <class EOS>
void noble(const EOS &eos, const C2P &cp, const Atmo &at_, Prim &p, Prim &sd, Cons &c,
           const Sym &g, Rep &r) { // c2p_2DNoble.hxx:275-594
  r.iters = 0;
  r.adjust = false;
  r.atmo = false;
  r.status = 0;
  const double dg = det(g), sdg = std::sqrt(dg);
  if (!sylvester(g, dg)) {
    r.fail(1);
    p.nan();
    c.nan();
    return;
  }
  const Sym gu = inv(g, dg);
  c.div(sdg);
  for (int i = 0; i < 3; ++i)
    sd.B[i] = c.B[i];
  double Su[3], Bl[3];
  ::mul(gu, c.S, Su);
  const double Ssq = dot(c.S, Su);
  ::mul(g, sd.B, Bl);
  const double Bsq = dot(Bl, sd.B);
  const double BiSi = dot(c.S, sd.B);
  double vsq_seed;
  if (cp.use_z) {
    double z[3], zl[3];
    for (int i = 0; i < 3; ++i)
      z[i] = sd.v[i] * sd.W;
    ::mul(g, z, zl);
    const double zsq = dot(zl, z);
    const double w = std::sqrt(1. + zsq);
    sd.W = w;
    vsq_seed = std::min(zsq / w / w, 1. - 1.e-15);
  } else {
    double vl[3];
    ::mul(g, sd.v, vl);
    const double vsq = dot(vl, sd.v);
    sd.W = 1. / std::sqrt(1. - vsq);
    vsq_seed = vsq;
  }
  if (!std::isfinite(c.D) || !std::isfinite(Ssq) || !std::isfinite(Bsq) ||
      !std::isfinite(BiSi) || !std::isfinite(c.DYe) || !std::isfinite(c.DEnt)) {
    r.fail(3);
    p.nan();
    c.nan();
    return;
  }
  if (Bsq > cp.Bsq_lim) {
    r.fail(8);
    p.nan();
    c.nan();
    return;
  }
  sd.rho = c.D / sd.W;
  double el = std::max({sd.eps, at_.eps});
  sd.press = eos.press_re(sd.rho, el, sd.Ye);
  const double Zs = (sd.rho + el * sd.rho + sd.press) * sd.W * sd.W;
  double x0 = std::fabs(Zs), x1 = vsq_seed, xo = x0;
  const double dv = 1. - 1.e-10, G = eos.gamma_noble(), Zmin = eos.rgrho.min;
  double errx = 1., df = 1., f = 1.;
  auto clamp = [&]() {
    if (x1 < 0.0)
      x1 = 0.0;
    else if (x1 >= 1.0)
      x1 = dv;
    if (x0 <= 0.0)
      x0 = std::fabs(x0) + Zmin;
    else if (x0 > 1e20)
      x0 = xo;
  };
  clamp();
  int k;
  for (k = 1; k <= cp.maxit; k++) {
    const double Z = x0, iZ = 1.0 / Z, V = x1;
    const double Sn = -(c.tau + c.D);
    const double pt = ((Z * (1.0 - V) - c.D * std::sqrt(1.0 - V)) * (G - 1.0) / (G));
    const double dpv = ((-Z + c.D / (2.0 * std::sqrt(1.0 - V))) * (G - 1.0) / G);
    const double dpz = ((1.0 - V) * (G - 1.0) / G);
    const double j00 = -2 * (V + BiSi * BiSi * iZ * iZ * iZ) * (Bsq + Z);
    const double j01 = -(Bsq + Z) * (Bsq + Z);
    const double j10 = -1.0 + dpz - BiSi * BiSi * iZ * iZ * iZ;
    const double j11 = -0.5 * Bsq + dpv;
    const double r0 = Ssq - V * (Bsq + Z) * (Bsq + Z) + BiSi * BiSi * iZ * iZ * (Bsq + Z + Z);
    const double r1 = -Sn - 0.5 * Bsq * (1.0 + V) + 0.5 * BiSi * BiSi * iZ * iZ - Z + pt;
    const double dj = (Bsq + Z) * (j10 * (Bsq + Z) + (Bsq - 2.0 * dpv) * (BiSi * BiSi * iZ * iZ + V * Z) * iZ);
    const double idj = 1.0 / dj;
    const double dx0 = -(j11 * r0 - j01 * r1) * idj;
    const double dx1 = -(-j10 * r0 + j00 * r1) * idj;
    df = -r0 * r0 - r1 * r1;
    f = -0.5 * (df);
    errx = 0.;
    xo = x0;
    x0 += dx0;
    x1 += dx1;
    clamp();
    errx = (x0 == 0.) ? std::fabs(dx0) : std::fabs(dx0 / x0);
    if (std::fabs(errx) <= cp.tol)
      break;
  }
  r.iters = k;
  if (std::fabs(errx) > cp.tol) {
    r.fail(9);
    c.mul(sdg);
    return;
  }
  if (!std::isfinite(f) || !std::isfinite(df))
    r.fail(10);
  const double W = 1.0 / std::sqrt(1.0 - x1);
  p.rho = c.D / W;
  velocity(x0, W, Bsq, BiSi, cp.use_z, p, c, gu, g);
  p.eps = (x0 / p.W / p.W / p.rho - 1.0) / G;
  p.Ye = c.DYe / c.D;
  p.press = eos.press_re(p.rho, p.eps, p.Ye);
  p.temp = eos.temp_re(p.rho, p.eps, p.Ye);
  p.ent = eos.kappa_re(p.rho, p.eps, p.Ye);
  for (int i = 0; i < 3; ++i)
    p.B[i] = c.B[i];
  efield(p, gu);
  if (p.rho <= 0.0) {
    r.fail(4);
    c.mul(sdg);
    return;
  }
  if (p.eps <= 0.0) {
    r.fail(5);
    c.mul(sdg);
    return;
  }
  c.DEnt = c.D * p.ent;
  if (p.rho < at_.cut) {
    r.status = 0;
    r.atmo = true;
    r.adjust = true;
    at_.set(p, c, g);
    return;
  }
  prim_floors(eos, cp, at_, p, c, g, r);
  if (r.adjust)
    from_prim(c, p, g);
  else
    c.mul(sdg);
}

// Brent bracketing solver with the contract of CarpetX Algo::brent as used
// at c2p_1DPalenzuela.hxx:380-417 (the same steps as the stand-in used to
// compile the reference; Brent 1973).
template <class Fn>
void brent_bracket(Fn &&f, double a, double b, int minbits, int maxit, int &it,
                   double &lo, double &hi) {
  const double eps = std::ldexp(1.0, -minbits);
  double fa = f(a), fb = f(b);
  it = 0;
  if (fa == 0) {
    lo = hi = a;
    return;
  }
  if (fb == 0) {
    lo = hi = b;
    return;
  }
  if (fa * fb > 0) {
    lo = std::min(a, b);
    hi = std::max(a, b);
    return;
  }
  if (std::fabs(fa) < std::fabs(fb)) {
    std::swap(a, b);
    std::swap(fa, fb);
  }
  double c = a, fc = fa, d = a;
  bool mflag = true;
  while (it < maxit) {
    if (std::fabs(b - a) <= eps * std::min(std::fabs(a), std::fabs(b)))
      break;
    ++it;
    double s;
    if (fa != fc && fb != fc)
      s = a * fb * fc / ((fa - fb) * (fa - fc)) + b * fa * fc / ((fb - fa) * (fb - fc)) +
          c * fa * fb / ((fc - fa) * (fc - fb));
    else
      s = b - fb * (b - a) / (fb - fa);
    const double delta = eps * std::fabs(b);
    const double q = (3 * a + b) / 4;
    const bool out = !((s > std::min(q, b)) && (s < std::max(q, b)));
    if (out || (mflag && std::fabs(s - b) >= std::fabs(b - c) / 2) ||
        (!mflag && std::fabs(s - b) >= std::fabs(c - d) / 2) ||
        (mflag && std::fabs(b - c) < delta) || (!mflag && std::fabs(c - d) < delta)) {
      s = (a + b) / 2;
      mflag = true;
    } else {
      mflag = false;
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
    if (std::fabs(fa) < std::fabs(fb)) {
      std::swap(a, b);
      std::swap(fa, fb);
    }
    if (fb == 0) {
      lo = hi = b;
      return;
    }
  }
  lo = std::min(a, b);
  hi = std::max(a, b);
}

template <class EOS>
void palenzuela(const EOS &eos, const C2P &cp, const Atmo &at_, Prim &p, Cons &c,
                const Sym &g, Rep &r) { // c2p_1DPalenzuela.hxx:306-556
  r.iters = 0;
  r.adjust = false;
  r.atmo = false;
  r.status = 0;
  const double dg = det(g), sdg = std::sqrt(dg);
  if (!sylvester(g, dg)) {
    r.fail(1);
    p.nan();
    c.nan();
    return;
  }
  const Sym gu = inv(g, dg);
  c.div(sdg);
  double Ssq = c.S[0] * (gu.xx * c.S[0] + gu.xy * c.S[1] + gu.xz * c.S[2]);
  Ssq += c.S[1] * (gu.xy * c.S[0] + gu.yy * c.S[1] + gu.yz * c.S[2]);
  Ssq += c.S[2] * (gu.xz * c.S[0] + gu.yz * c.S[1] + gu.zz * c.S[2]);
  double Bl[3];
  ::mul(g, c.B, Bl);
  const double Bsq = dot(Bl, c.B);
  const double BiSi = c.B[0] * c.S[0] + c.B[1] * c.S[1] + c.B[2] * c.S[2];
  if (!std::isfinite(c.D) || !std::isfinite(Ssq) || !std::isfinite(Bsq) ||
      !std::isfinite(BiSi) || !std::isfinite(c.DYe) || !std::isfinite(c.DEnt)) {
    r.fail(3);
    p.nan();
    c.nan();
    return;
  }
  if (Bsq > cp.Bsq_lim) {
    r.fail(8);
    p.nan();
    c.nan();
    return;
  }
  const int minbits = int(std::abs(std::log(cp.tol)) / std::log(2.0));
  const double tol0 = std::ldexp(double(1.0), -minbits);
  const double q = c.tau / c.D, rr = Ssq / std::pow(c.D, 2), s = Bsq / c.D,
               t = BiSi / std::pow(c.D, 3. / 2.);
  auto x2prim_W = [&](double x, double &Wo) {
    double Wm2 = 1.0 - (x * x * rr + (2.0 * x + s) * t * t) / (x * x * (x + s) * (x + s));
    Wm2 = std::fmin(std::fmax(Wm2, 1e-10), 1);
    Wo = std::pow(Wm2, -0.5);
  };
  auto fn = [&](double x) { // funcRoot_1DPalenzuela (:260-304)
    double W;
    x2prim_W(x, W);
    const double rho = c.D / W, ye = c.DYe / c.D;
    double e = W - 1.0 + (1.0 - W * W) * x / W + W * (q - s + t * t / (2 * x * x) + s / (2 * W * W));
    if (cp.use_temp) {
      e = std::max(e, at_.eps);
      e = std::min(e, eos.rgeps.max);
    }
    const double P = eos.press_re(rho, e, ye);
    return (x - (1.0 + e + P / rho) * W);
  };
  double a = std::max(1e-10, 1.0 + q - s), b = 2.0 + 2.0 * q - s;
  if (fn(a) * fn(b) > 0)
    b = 3.0 + 3.0 * q - 1.5 * s;
  double r0, r1;
  brent_bracket(fn, a, b, minbits, cp.maxit, r.iters, r0, r1);
  const double x = 0.5 * (r0 + r1);
  double W;
  x2prim_W(x, W);
  p.rho = c.D / W;
  p.eps = W - 1.0 + (1.0 - W * W) * x / W + W * (q - s + t * t / (2 * x * x) + s / (2.0 * W * W));
  if (cp.use_temp) {
    p.eps = std::max(p.eps, at_.eps);
    p.eps = std::min(p.eps, eos.rgeps.max);
  }
  velocity(x * p.rho * W, W, Bsq, BiSi, cp.use_z, p, c, gu, g);
  p.Ye = c.DYe / c.D;
  p.press = eos.press_re(p.rho, p.eps, p.Ye);
  p.temp = eos.temp_re(p.rho, p.eps, p.Ye);
  p.ent = eos.kappa_re(p.rho, p.eps, p.Ye);
  for (int i = 0; i < 3; ++i)
    p.B[i] = c.B[i];
  efield(p, gu);
  if (p.rho <= 0.0) {
    r.fail(4);
    c.mul(sdg);
    return;
  }
  if (p.eps <= 0.0) {
    r.fail(5);
    c.mul(sdg);
    return;
  }
  if (std::abs(r0 - r1) > tol0 * std::min(std::abs(r0), std::abs(r1))) {
    Cons ck;
    from_prim(ck, p, g);
    ck.div(sdg);
    const double sm = 1e-50;
    const double me = std::sqrt(std::max({std::pow((ck.D - c.D) / (c.D + sm), 2.0),
                                          std::pow((ck.S[0] - c.S[0]) / (c.S[0] + sm), 2.0),
                                          std::pow((ck.S[1] - c.S[1]) / (c.S[1] + sm), 2.0),
                                          std::pow((ck.S[2] - c.S[2]) / (c.S[2] + sm), 2.0),
                                          std::pow((ck.tau - c.tau) / (c.tau + sm), 2.0)}));
    if (me > cp.cons_err) {
      r.fail(9);
      c.mul(sdg);
      return;
    }
  }
  c.DEnt = c.D * p.ent;
  if (p.rho < at_.cut) {
    r.status = 0;
    r.atmo = true;
    r.adjust = true;
    at_.set(p, c, g);
    return;
  }
  prim_floors(eos, cp, at_, p, c, g, r);
  if (r.adjust)
    from_prim(c, p, g);
  else
    c.mul(sdg);
}

template <class EOS>
void bh_interior(const EOS &eos, const C2P &cp, const Atmo &at_, bool limiting, Prim &p,
                 Cons &c, const Sym &g) { // c2p.hxx:218-328
  const double wl = std::sqrt(1.0 + cp.vwlim_BH * cp.vwlim_BH), vl = cp.vwlim_BH / wl;
  if (limiting) {
    bool re = false;
    if (p.rho > cp.rho_BH) {
      p.rho = cp.rho_BH;
      re = true;
    }
    if (p.eps > cp.eps_BH) {
      p.eps = cp.eps_BH;
      re = true;
    }
    const double sv = std::sqrt((p.W * p.W - 1.0)) / p.W;
    if (sv > vl) {
      for (int i = 0; i < 3; ++i)
        p.v[i] *= vl / sv;
      p.W = wl;
      re = true;
    }
    if (re) {
      p.temp = eos.temp_re(p.rho, p.eps, p.Ye);
      p.press = eos.press_re(p.rho, p.eps, p.Ye);
      p.ent = eos.kappa_re(p.rho, p.eps, p.Ye);
      from_prim(c, p, g);
    }
    return;
  }
  p.rho = cp.rho_BH;
  p.eps = cp.eps_BH;
  p.Ye = at_.ye;
  p.temp = eos.temp_re(p.rho, p.eps, p.Ye);
  p.press = eos.press_re(p.rho, p.eps, p.Ye);
  p.ent = eos.kappa_re(p.rho, p.eps, p.Ye);
  const double dg = det(g);
  const Sym gu = inv(g, dg);
  const double Z = (p.rho * (1.0 + p.eps) + p.press) * wl * wl;
  double Bl[3];
  ::mul(g, p.B, Bl);
  const double Bsq = dot(Bl, p.B);
  double ml[3], mu[3];
  for (int i = 0; i < 3; ++i)
    ml[i] = c.S[i] / std::sqrt(dg);
  ::mul(gu, ml, mu);
  const double So = std::sqrt(dot(ml, mu)) + 1e-50;
  const double BE = dot(ml, p.B) / So;
  const double Sn = std::sqrt(((Z + Bsq) * (Z + Bsq) * vl * vl) /
                              (1.0 + BE * BE * (2.0 * Z + Bsq) / (Z * Z)));
  for (int i = 0; i < 3; ++i) {
    ml[i] *= Sn / So;
    mu[i] *= Sn / So;
  }
  for (int i = 0; i < 3; ++i) {
    p.v[i] = mu[i] / (Z + Bsq);
    p.v[i] += BE * Sn * p.B[i] / (Z * (Z + Bsq));
  }
  p.W = wl;
  from_prim(c, p, g);
}

template <class EOS> Atmo atmosphere(const EOS &eos, double x, double y, double z) {
  const axb_params &P = g_p; // con2prim.cxx:81-133
  const double r = std::sqrt(x * x + y * y + z * z);
  double rho = (r > P.r_atmo) ? (P.rho_abs_min * std::pow((P.r_atmo / r), P.n_rho_atmo))
                              : P.rho_abs_min;
  rho = std::max(eos.rgrho.min, rho);
  double press, eps, temp = 0.0;
  if (P.thermal_eos_atmo) {
    if (P.use_press_atmo) {
      press = (r > P.r_atmo) ? (P.p_atmo * std::pow(P.r_atmo / r, P.n_press_atmo)) : P.p_atmo;
      press = std::max(eos.press_rt(rho, eos.rgtemp.min, P.Ye_atmo), press);
      eps = eos.eps_rp(rho, press, P.Ye_atmo);
      temp = eos.temp_re(rho, eps, P.Ye_atmo);
    } else {
      temp = (r > P.r_atmo) ? (P.t_atmo * std::pow(P.r_atmo / r, P.n_temp_atmo)) : P.t_atmo;
      temp = std::max(eos.rgtemp.min, temp);
      press = eos.press_rt(rho, temp, P.Ye_atmo);
      eps = eos.eps_rt(rho, temp, P.Ye_atmo);
    }
  } else {
    eps = g_poly.sed_gm1(g_poly.gm1_rho(rho));
    eps = std::min(std::max(eos.rgeps.min, eps), eos.rgeps.max);
    press = eos.press_re(rho, eps, P.Ye_atmo);
  }
  const double ent = eos.kappa_re(rho, eps, P.Ye_atmo);
  return Atmo{rho, eps, P.Ye_atmo, press, temp, ent, rho * (1 + P.atmo_tol)};
}

template <class EOS>
void run_solver(int which, const EOS &eos, const C2P &cp, const Atmo &a, Prim &p, Prim &sd,
                Cons &c, const Sym &g, Rep &r) {
  if (which == AXB_C2P_NOBLE)
    noble(eos, cp, a, p, sd, c, g, r);
  else if (which == AXB_C2P_PALENZUELA)
    palenzuela(eos, cp, a, p, c, g, r);
}

template <class EOS> void con2prim(const EOS &eos) {
  const axb_params &P = g_p;
  if (P.use_entropy_fix || P.use_mask)
    throw Fail("entropy fix and masks are not restated");
  const C2P cp = c2p_params();
  const double *alp = need("alp");
  const double *gg[6] = {need("gxx"), need("gxy"), need("gxz"), need("gyy"), need("gyz"), need("gzz")};
  double *D = need("dens"), *S[3] = {need("momx"), need("momy"), need("momz")},
         *tau = need("tau"), *DYe = need("DYe"), *DEnt = need("DEnt");
  double *dB[3] = {need("dBx"), need("dBy"), need("dBz")};
  double *rho = need("rho"), *eps = need("eps"), *Ye = need("Ye"), *press = need("press"),
         *temp = need("temperature"), *ent = need("entropy");
  double *vel[3] = {need("velx"), need("vely"), need("velz")};
  double *Bv[3] = {need("Bvecx"), need("Bvecy"), need("Bvecz")};
  double *sr = need("saved_rho"), *sv[3] = {need("saved_velx"), need("saved_vely"), need("saved_velz")},
         *se = need("saved_eps"), *sy = need("saved_Ye");
  double *zv[3] = {F("zvec_x"), F("zvec_y"), F("zvec_z")};
  double *svv[3] = {F("svec_x"), F("svec_y"), F("svec_z")};
  double *flag = need("con2prim_flag");
  loop(1, 1, 1, [&](int i, int j, int k) {
    const long long I = at(i, j, k);
    const double x = g_box.xmin[0] + (i - g_box.ng + 0.5) * g_box.dx[0];
    const double y = g_box.xmin[1] + (j - g_box.ng + 0.5) * g_box.dx[1];
    const double z = g_box.xmin[2] + (k - g_box.ng + 0.5) * g_box.dx[2];
    const Atmo atm = atmosphere(eos, x, y, z);
    auto v2c = [&](const double *f) {
      double s = 0.0;
      for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
          for (int di = 0; di < 2; ++di)
            s += f[I + di + g_box.sy * dj + g_box.sz * dk];
      return s / 8.0;
    };
    const double a = v2c(alp);
    const Sym g{v2c(gg[0]), v2c(gg[1]), v2c(gg[2]), v2c(gg[3]), v2c(gg[4]), v2c(gg[5])};
    double mask = 1.0;
    const double dg = det(g), sdg = std::sqrt(dg);
    double vu[3] = {sv[0][I], sv[1][I], sv[2][I]}, vl[3];
    ::mul(g, vu, vl);
    const double vsq = dot(vl, vu);
    double zsq;
    if (vsq >= 1.0) {
      const double wlim = std::sqrt(1.0 + P.vw_lim * P.vw_lim), vlim = P.vw_lim / wlim;
      for (int q = 0; q < 3; ++q) {
        vu[q] *= vlim / std::sqrt(vsq);
        vl[q] *= vlim / std::sqrt(vsq);
      }
      zsq = P.vw_lim * P.vw_lim;
    } else {
      zsq = vsq / (1.0 - vsq);
    }
    double wlor = std::sqrt(1.0 + zsq);
    Cons c{D[I], {S[0][I], S[1][I], S[2][I]}, tau[I], DYe[I], DEnt[I], {dB[0][I], dB[1][I], dB[2][I]}};
    const double Bu[3] = {c.B[0] / sdg, c.B[1] / sdg, c.B[2] / sdg};
    Prim p;
    p.nan();
    Prim sd;
    sd.rho = sr[I];
    sd.eps = se[I];
    sd.Ye = sy[I];
    {
      double e = se[I];
      sd.press = eos.press_re(sr[I], e, sy[I]);
    }
    sd.temp = temp[I];
    sd.ent = 0.0;
    for (int q = 0; q < 3; ++q)
      sd.v[q] = vu[q], sd.B[q] = Bu[q], sd.E[q] = 0.0;
    sd.W = wlor;
    bool ok = true, call = true;
    int code = AXB_C2P_INIT;
    if (c.D <= sdg * atm.cut) {
      for (int q = 0; q < 3; ++q)
        p.B[q] = Bu[q];
      atm.set(p, c, g);
      atm.set(sd);
      code = AXB_C2P_ATMO;
      call = false;
    }
    if (a < P.alp_thresh)
      mask = 0.0;
    if (P.excise && mask != 1.0) {
      double e = sd.eps;
      sd.ent = eos.kappa_re(sd.rho, e, sd.Ye);
      bh_interior(eos, cp, atm, false, sd, c, g);
      p = sd;
      call = false;
    }
    cons_floors(c, g);
    if (call) {
      Rep r1, r2;
      code = AXB_C2P_PRIME;
      run_solver(P.c2p_prime, eos, cp, atm, p, sd, c, g, r1);
      if (r1.failed()) {
        code = AXB_C2P_SECOND;
        run_solver(P.c2p_second, eos, cp, atm, p, sd, c, g, r2);
      }
      if (r1.failed() && r2.failed()) {
        ok = false;
        code = AXB_C2P_FAIL;
        if (mask != 1.0) {
          bh_interior(eos, cp, atm, false, sd, c, g);
          p = sd;
        } else {
          for (int q = 0; q < 3; ++q) {
            c.B[q] = sdg * Bu[q];
            p.B[q] = Bu[q];
          }
          atm.set(p, c, g);
        }
      }
      if (mask != 1.0 && ok)
        bh_interior(eos, cp, atm, true, p, c, g);
    }
    flag[I] = code;
    rho[I] = p.rho;
    eps[I] = p.eps;
    Ye[I] = p.Ye;
    press[I] = p.press;
    temp[I] = p.temp;
    ent[I] = p.ent;
    for (int q = 0; q < 3; ++q)
      vel[q][I] = p.v[q], Bv[q][I] = p.B[q];
    wlor = p.W;
    for (int q = 0; q < 3; ++q) {
      if (zv[q])
        zv[q][I] = wlor * p.v[q];
      if (svv[q])
        svv[q][I] = (p.rho + p.rho * p.eps + p.press) * wlor * wlor * p.v[q];
    }
    D[I] = c.D;
    for (int q = 0; q < 3; ++q)
      S[q][I] = c.S[q], dB[q][I] = c.B[q];
    tau[I] = c.tau;
    DYe[I] = c.DYe;
    DEnt[I] = c.DEnt;
    sr[I] = rho[I];
    for (int q = 0; q < 3; ++q)
      sv[q][I] = vel[q][I];
    se[I] = eps[I];
    sy[I] = Ye[I];
  });
}

template <class Fn> void with_eos(Fn &&fn) {
  if (g_eos_kind == 0)
    fn(g_ideal);
  else if (g_eos_kind == 1)
    fn(g_tab);
  else
    throw Fail("no EOS set");
}

} // namespace

// ---------------------------------------------------------------------------
// C ABI (same entry points as oracle/refshim/axref_harness.cpp)
// ---------------------------------------------------------------------------
extern "C" {

const char *ora_last_error(void) { return g_err; }

int ora_bind(const char *name, double *ptr) {
  for (int i = 0; i < kNFields; ++i)
    if (!std::strcmp(kNames[i], name)) {
      g_f[i] = ptr;
      return 0;
    }
  return 1;
}

int ora_setup(const axb_box *b, const axb_params *p, int) {
  for (int d = 0; d < 3; ++d) {
    g_box.n[d] = b->n[d];
    g_box.dx[d] = b->dx[d];
    g_box.xmin[d] = b->xmin[d];
  }
  g_box.ng = b->ng;
  g_box.sy = b->sy;
  g_box.sz = b->sz;
  g_p = *p;
  g_ext_c = g_ext_v = 0;
  return 0;
}

void ora_set_ext(int ext_c, int ext_v) {
  g_ext_c = ext_c;
  g_ext_v = ext_v;
}

int ora_eos_idealgas(double gamma, double umass, double rho_min, double rho_max,
                     double eps_min, double eps_max, double ye_min, double ye_max,
                     double poly_gamma, double poly_k) {
  // eos_3p_idealgas::init (eos_3p_idealgas.hxx:124-142)
  g_ideal.gamma = gamma;
  g_ideal.gm1 = gamma - 1;
  g_ideal.inv_gamma = 1 / gamma;
  g_ideal.rgeps = Range{eps_min, eps_max};
  if (gamma > 2)
    g_ideal.rgeps.max = std::min(g_ideal.rgeps.max, 1 / (gamma * (gamma - 2)));
  g_ideal.rgrho = Range{rho_min, rho_max};
  g_ideal.rgye = Range{ye_min, ye_max};
  g_ideal.temp_over_eps = g_ideal.gm1 * umass;
  g_ideal.rgtemp = Range{g_ideal.temp_over_eps * g_ideal.rgeps.min,
                         g_ideal.temp_over_eps * g_ideal.rgeps.max};
  // eos_1p_polytropic::init (eos_1p_polytropic.hxx:57-67)
  g_poly.k = poly_k;
  g_poly.gamma = poly_gamma;
  g_poly.n = 1.0 / (poly_gamma - 1.0);
  g_poly.np1 = g_poly.n + 1;
  g_poly.invn = 1.0 / g_poly.n;
  g_poly.rho_p = std::pow(poly_k, -g_poly.n);
  g_eos_kind = 0;
  return 0;
}

int ora_eos_tabulated(int nrho, int ntemp, int nye, const double *logrho,
                      const double *logtemp, const double *yes, const double *table,
                      double energy_shift, double poly_gamma, double poly_k) {
  Table &t = g_tab.t;
  t.n[0] = nrho;
  t.n[1] = ntemp;
  t.n[2] = nye;
  t.x[0].assign(logrho, logrho + nrho);
  t.x[1].assign(logtemp, logtemp + ntemp);
  t.x[2].assign(yes, yes + nye);
  const size_t total = size_t(nrho) * ntemp * nye;
  t.y.assign(table, table + total * Table::NV);
  for (int d = 0; d < 3; ++d) {
    t.dx[d] = t.x[d][1] - t.x[d][0];
    t.idx[d] = 1. / t.dx[d];
  }
  g_tab.shift = energy_shift;
  g_tab.rgrho = Range{std::exp(t.x[0].front()), std::exp(t.x[0].back())};
  g_tab.rgtemp = Range{std::exp(t.x[1].front()), std::exp(t.x[1].back())};
  g_tab.rgye = Range{t.x[2].front(), t.x[2].back()};
  // compute_eps_range_full_table (:352-367) reads the block starting at
  // EPS * total of the variable-fastest table, as the reference does
  double emin = std::numeric_limits<double>::max(), emax = std::numeric_limits<double>::lowest();
  for (size_t i = 0; i < total; ++i) {
    const double v = std::exp(t.y[Tab::EPS * total + i]) - energy_shift;
    emin = std::fmin(emin, v);
    emax = std::fmax(emax, v);
  }
  g_tab.rgeps = Range{std::fmax(emin, 1e-15), emax};
  g_poly.k = poly_k;
  g_poly.gamma = poly_gamma;
  g_poly.n = 1.0 / (poly_gamma - 1.0);
  g_poly.np1 = g_poly.n + 1;
  g_poly.invn = 1.0 / g_poly.n;
  g_poly.rho_p = std::pow(poly_k, -g_poly.n);
  g_eos_kind = 1;
  return 0;
}

void ora_eos_tab_ranges(double *o) {
  o[0] = g_tab.rgrho.min, o[1] = g_tab.rgrho.max;
  o[2] = g_tab.rgtemp.min, o[3] = g_tab.rgtemp.max;
  o[4] = g_tab.rgye.min, o[5] = g_tab.rgye.max;
  o[6] = g_tab.rgeps.min, o[7] = g_tab.rgeps.max;
}

int ora_fluxes(void) {
  return guarded([] {
    if (g_p.recon_type != AXB_RECVAR_V)
      throw Fail("only v_vec reconstruction is restated");
    with_eos([](const auto &eos) {
      for (int d = 0; d < 3; ++d)
        calc_flux(eos, d);
    });
    calc_aux();
  });
}
int ora_sources(void) { return guarded([] { source_terms(); }); }
int ora_rhs(void) { return guarded([] { rhs(); }); }
int ora_bstag(void) { return guarded([] { bstag(); }); }
int ora_dB(void) { return guarded([] { dB_from_stag(); }); }
int ora_c2p(void) {
  return guarded([] { with_eos([](const auto &eos) { con2prim(eos); }); });
}

void ora_reconstruct(int method, const double *v, const double *press, const double *vel,
                     int is_rho, int, double *out) {
  recon_face(method, v, press, vel, is_rho != 0, out);
}

void ora_eigen(const double *in, double *lam) {
  const double alp = in[0], be = in[1], u = in[2];
  for (int f = 0; f < 2; ++f) {
    const double vel = in[3 + f], rho = in[5 + f], cs2 = in[7 + f], w = in[9 + f],
                 h = in[11 + f], bsq = in[13 + f];
    const double a0 = (bsq + cs2 * h * rho) * (p2(be) - p2(alp) * u) -
                      (-1 + cs2) * h * rho * p2(be - alp * vel) * p2(w);
    const double a1 = 2 * be * (bsq + cs2 * h * rho) - 2 * (-1 + cs2) * h * rho * (be - alp * vel) * p2(w);
    const double a2 = bsq + h * rho * (cs2 + p2(w) - cs2 * p2(w));
    double d = p2(a1) - 4 * a2 * a0;
    if (d < 0)
      d = 0;
    lam[4 * f + 0] = lam[4 * f + 1] = ((-a1 + std::sqrt(d)) / (2 * a2)) / alp;
    lam[4 * f + 2] = lam[4 * f + 3] = ((-a1 - std::sqrt(d)) / (2 * a2)) / alp;
  }
}

double ora_riemann(int flux_type, const double *l, double uL, double uR, double fL, double fR) {
  if (flux_type == AXB_FLUX_HLLE) { // fluxes.hxx:32-49
    const double cmax = std::max({0.0, l[0], l[1], l[2], l[3], l[4], l[5], l[6], l[7]});
    const double cmin = std::min({0.0, l[0], l[1], l[2], l[3], l[4], l[5], l[6], l[7]});
    return (cmax * fL - cmin * fR + cmax * cmin * (uR - uL)) / (cmax - cmin);
  }
  const double cm = std::max({0.0, std::fabs(l[0]), std::fabs(l[1]), std::fabs(l[2]), std::fabs(l[3]),
                              std::fabs(l[4]), std::fabs(l[5]), std::fabs(l[6]), std::fabs(l[7])});
  return 0.5 * ((fL + fR) - cm * (uR - uL)); // fluxes.hxx:20-29
}

void ora_prim2con(const double *g6, const double *prim, double *cons) {
  // prim2con.hxx:38-83 (W from the velocity)
  const Sym g{g6[0], g6[1], g6[2], g6[3], g6[4], g6[5]};
  const double sd = std::sqrt(det(g));
  const double v[3] = {prim[1], prim[2], prim[3]}, B[3] = {prim[8], prim[9], prim[10]};
  double vl[3], Bl[3];
  ::mul(g, v, vl);
  const double W = 1.0 / std::sqrt(1.0 - dot(vl, v));
  ::mul(g, B, Bl);
  const double bst = W * dot(B, vl);
  double bl[3];
  for (int i = 0; i < 3; ++i)
    bl[i] = Bl[i] / W + bst * vl[i];
  const double bs2 = (dot(B, Bl) + bst * bst) / (W * W);
  const double rho = prim[0], eps = prim[4], press = prim[5];
  cons[0] = sd * rho * W;
  const double h = W * W * (rho * (1.0 + eps) + press + bs2);
  for (int i = 0; i < 3; ++i)
    cons[1 + i] = sd * (h * vl[i] - bst * bl[i]);
  cons[4] = sd * (h - (press + 0.5 * bs2) - bst * bst) - cons[0];
  cons[6] = cons[0] * prim[7];
  for (int i = 0; i < 3; ++i)
    cons[7 + i] = sd * B[i];
  cons[5] = prim[6] * cons[0];
}

int ora_c2p_point(int solver, double *cons, const double *g6, const double *seed,
                  const double *atmo, double *prim, int *rep3) {
  return guarded([&] {
    with_eos([&](const auto &eos) {
      const Atmo a{atmo[0], atmo[1], atmo[2], atmo[3], atmo[4], atmo[5], atmo[6]};
      const Sym g{g6[0], g6[1], g6[2], g6[3], g6[4], g6[5]};
      Cons c{cons[0], {cons[1], cons[2], cons[3]}, cons[4], cons[5], cons[6], {cons[7], cons[8], cons[9]}};
      Prim p;
      p.nan();
      Rep r;
      const C2P cp = c2p_params();
      if (solver == AXB_C2P_NOBLE) {
        const double sdg = std::sqrt(det(g));
        Prim sd;
        sd.rho = seed[0];
        sd.eps = seed[1];
        sd.Ye = seed[2];
        sd.press = seed[3];
        sd.temp = seed[4];
        sd.ent = seed[5];
        for (int q = 0; q < 3; ++q)
          sd.v[q] = seed[6 + q], sd.B[q] = c.B[q] / sdg, sd.E[q] = 0;
        sd.W = 1.0;
        noble(eos, cp, a, p, sd, c, g, r);
      } else {
        palenzuela(eos, cp, a, p, c, g, r);
      }
      cons[0] = c.D;
      for (int q = 0; q < 3; ++q)
        cons[1 + q] = c.S[q], cons[7 + q] = c.B[q];
      cons[4] = c.tau;
      cons[5] = c.DYe;
      cons[6] = c.DEnt;
      const double pv[16] = {p.rho, p.eps, p.Ye, p.press, p.temp, p.ent, p.v[0], p.v[1],
                             p.v[2], p.W, p.B[0], p.B[1], p.B[2], p.E[0], p.E[1], p.E[2]};
      for (int q = 0; q < 16; ++q)
        prim[q] = pv[q];
      rep3[0] = r.status;
      rep3[1] = r.iters;
      rep3[2] = r.adjust;
    });
  });
}

double ora_eos_tab_query(int which, double rho, double x, double ye, double *eps_io) {
  double e = x, r = 0;
  switch (which) {
  case 0: r = g_tab.press_re(rho, e, ye); break;
  case 1: r = g_tab.temp_re(rho, e, ye); break;
  case 2: r = g_tab.csnd_re(rho, e, ye); break;
  case 3: r = g_tab.kappa_re(rho, e, ye); break;
  case 4: r = g_tab.eps_rt(rho, x, ye); break;
  case 5: r = g_tab.press_rt(rho, x, ye); break;
  case 6: r = g_tab.entropy_rt(rho, x, ye); break;
  }
  if (eps_io)
    *eps_io = e;
  return r;
}

} // extern "C"
