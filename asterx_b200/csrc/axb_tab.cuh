// Tabulated 3D EOS on the device (EOSX eos_3p_tabulated3d).
//
//   queries        EOSX/src/eos_3p_tabulated3d/eos_3p_tabulated3d.hxx:197-350
//   interpolation  EOSX/src/utils/eos_linear_interp_ND.hxx:50-206 (uniform
//                  axes, index clamped to [0, n-2], linear along ln rho, then
//                  ln T, then Ye)
//   T inversion    the root of the interpolant, found exactly (logtemp_root);
//                  Brent's zero finder (EOSX/src/utils/eos_brent.hxx:7-170)
//                  where the table is not monotonic in T
//
// Layout: only the four variables the hot path reads are kept, interleaved
// per node as (ln P, ln(eps + shift), s, cs^2) -- variables 0, 1, 2 and 4 of
// the reference's 19 -- so that one trilinear corner is one 32-byte DRAM
// sector; the 200 x 100 x 60 synthetic table is 38 MB and stays resident in
// the 126 MB L2 across a step.  The values are copied bit for bit.
#pragma once

#include "axb_eos.cuh"

namespace axb {

constexpr int TAB_NV = 4;
enum { TAB_PRESS = 0, TAB_EPS = 1, TAB_S = 2, TAB_CS2 = 3 };
// Iteration cap of the temperature root find.  The reference's loop has no
// cap; Brent's method needs at most about (log2(interval / tol))^2 ~ 2500
// steps here and in practice a few dozen.  A capped query sets
// AXB_EW_ROOT_CAP in the status word instead of spinning.
constexpr int TAB_BRENT_MAXIT = 10000;

struct EosTab {
  int n[3];
  const double *x[3]; // axis values (device)
  double idx[3];      // 1 / (x[d][1] - x[d][0])
  double x0[3], xlast[3];
  const double *y; // TAB_NV values per node, node = i + n0*(j + n1*k)
  double shift;
  Range rgrho, rgye, rgtemp, rgeps;
  unsigned int *err; // status error word (device descriptor only), or null

  static constexpr bool kTabulated = true;

  // The cell of the uniform axis d holding xin, clamped to [0, n - 2]
  // (eos_linear_interp_ND.hxx:50-65).  The clamps act on the floating-point
  // position before it becomes an integer, so a NaN query (the logarithm of
  // a non-positive temperature that press_from_valid_rho_temp_ye takes
  // before clamping) and an infinite one map to an end cell instead of an
  // undefined conversion; finite queries are unchanged.
  AXB_HD int find(int d, double xin) const {
    const double xL = xin - x0[d];
    if (!(xL > 0))
      return 0;
    const double t = xL * idx[d];
    if (!(t < double(n[d] - 2)))
      return n[d] - 2;
    return static_cast<int>(t);
  }
  AXB_HD static double lin(double A, double B, double xA, double xB, double xv) {
    const double lam = (xv - xA) / (xB - xA);
    return (B - A) * lam + A;
  }
  AXB_HD double interp(int var, double a, double b, double c) const {
    const int i = find(0, a), j = find(1, b), k = find(2, c);
    double Bk[2];
#pragma unroll
    for (int o2 = 0; o2 < 2; ++o2) {
      double Aj[2];
#pragma unroll
      for (int o1 = 0; o1 < 2; ++o1) {
        const long long base = i + (long long)n[0] * ((j + o1) + (long long)n[1] * (k + o2));
        Aj[o1] = lin(y[TAB_NV * base + var], y[TAB_NV * (base + 1) + var], x[0][i],
                     x[0][i + 1], a);
      }
      Bk[o2] = lin(Aj[0], Aj[1], x[1][j], x[1][j + 1], b);
    }
    return lin(Bk[0], Bk[1], x[2][k], x[2][k + 1], c);
  }

  template <class Fn>
  AXB_HD static double zero_brent(double a, double b, double t, const Fn &f,
                                  bool &capped) {
    double sa = a, sb = b, fa = f(sa), fb = f(sb);
    double c = sa, fc = fa, e = sb - sa, d = e;
    const double macheps = 2.220446049250313e-16;
    capped = true;
    for (int it = 0; it < TAB_BRENT_MAXIT; ++it) {
      if (fabs(fc) < fabs(fb)) {
        sa = sb;
        sb = c;
        c = sa;
        fa = fb;
        fb = fc;
        fc = fa;
      }
      const double tol = 2.0 * macheps * fabs(sb) + t;
      const double m = 0.5 * (c - sb);
      if (fabs(m) <= tol || fb == 0.0) {
        capped = false;
        break;
      }
      if (fabs(e) < tol || fabs(fa) <= fabs(fb)) {
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
        if (2.0 * p < 3.0 * m * q - fabs(tol * q) && p < fabs(0.5 * s * q)) {
          d = p / q;
        } else {
          e = m;
          d = e;
        }
      }
      sa = sb;
      fa = fb;
      if (tol < fabs(d))
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

  // logtemp_from_valid_rho_eps_ye (:197-228): clamps eps in place.
  AXB_HD double logtemp(double rho, double &eps, double ye) const {
    const double r = fmin(fmax(rho, rgrho.min), rgrho.max);
    eps = fmax(eps + shift, rgeps.min + shift) - shift;
    const double lrho = log(r);
    const double leps = log(eps + shift);
    const double vmin = interp(TAB_EPS, lrho, x0[1], ye);
    const double vmax = interp(TAB_EPS, lrho, xlast[1], ye);
    if (leps <= vmin) {
      eps = exp(vmin) - shift;
      return x0[1];
    }
    if (leps >= vmax) {
      eps = exp(vmax) - shift;
      return xlast[1];
    }
    return logtemp_root(lrho, leps, ye, vmin, vmax);
  }

  // The root in ln T of leps = interp(EPS, lrho, ln T, ye).  The
  // interpolant is linear in ln T within each cell of the T axis (the
  // trilinear scheme interpolates along ln T between the two T nodes of the
  // cell), so the root is found exactly: a bisection over the nodes' values
  // (which grow with T for a thermodynamic table) locates the cell, and the
  // linear equation of that cell gives the root.  The reference runs Brent's
  // method on the whole axis to 1e-14 (eos_3p_tabulated3d.hxx:219-225,
  // eos_brent.hxx); both land on the same root of the same interpolant,
  // here to rounding.  Where the node values are not increasing around the
  // root, the reference's Brent search is run instead.
  AXB_HD double logtemp_root(double lrho, double leps, double ye, double vlo, double vhi) const {
    // vlo = interp at node 0 < leps < vhi = interp at the last node.
    // The bisection evaluates the interpolant at temperature nodes, where it
    // is the bilinear interpolant in (ln rho, Ye) of that node's four
    // values: the rho and Ye cells and weights are found once, and each step
    // reads four values (interp's own arithmetic with the temperature weight
    // zero)
    const int i = find(0, lrho), k = find(2, ye);
    const double lam_r = (lrho - x[0][i]) / (x[0][i + 1] - x[0][i]);
    const double lam_y = (ye - x[2][k]) / (x[2][k + 1] - x[2][k]);
    auto at_node = [&](int jn) {
      double A[2];
#pragma unroll
      for (int o2 = 0; o2 < 2; ++o2) {
        const long long base = i + (long long)n[0] * (jn + (long long)n[1] * (k + o2));
        const double y0 = y[TAB_NV * base + TAB_EPS], y1 = y[TAB_NV * (base + 1) + TAB_EPS];
        A[o2] = (y1 - y0) * lam_r + y0;
      }
      return (A[1] - A[0]) * lam_y + A[0];
    };
    int lo = 0, hi = n[1] - 1;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      const double vm = at_node(mid);
      if (vm <= leps) {
        lo = mid;
        vlo = vm;
      } else {
        hi = mid;
        vhi = vm;
      }
    }
    // the cell [x_lo, x_lo+1]: interp = c0 + c1 * lambda, lambda in [0, 1]
    const double xa = x[1][lo], xb = x[1][lo + 1];
    double c[2][2]; // [T end][Ye end] after the interpolation along ln rho
#pragma unroll
    for (int o2 = 0; o2 < 2; ++o2)
#pragma unroll
      for (int o1 = 0; o1 < 2; ++o1) {
        const long long base =
            i + (long long)n[0] * ((lo + o1) + (long long)n[1] * (k + o2));
        const double y0 = y[TAB_NV * base + TAB_EPS], y1 = y[TAB_NV * (base + 1) + TAB_EPS];
        c[o1][o2] = (y1 - y0) * lam_r + y0; // lin along ln rho, its weight found once
      }
    const double e0 = (c[0][1] - c[0][0]) * lam_y + c[0][0]; // at x_lo
    const double e1 = (c[1][1] - c[1][0]) * lam_y + c[1][0]; // at x_lo+1
    if (!(vlo <= leps && leps <= vhi) || !(e1 > e0)) {
      bool capped;
      const double lt = zero_brent(
          x0[1], xlast[1], 1.e-14,
          [&](double l) { return leps - interp(TAB_EPS, lrho, l, ye); }, capped);
#ifdef __CUDA_ARCH__
      if (capped && err)
        atomicOr(err, AXB_EW_ROOT_CAP);
#endif
      return lt;
    }
    const double lam = fmin(fmax((leps - e0) / (e1 - e0), 0.0), 1.0);
    return xa + lam * (xb - xa);
  }
  AXB_HD double lr_clamped(double rho) const {
    return log(fmin(fmax(rho, rgrho.min), rgrho.max));
  }
  AXB_HD double lt_clamped(double temp) const {
    return log(fmin(fmax(temp, rgtemp.min), rgtemp.max));
  }
  AXB_HD double press_over_rho(double rho, double &eps, double ye) const {
    return press_from_valid_rho_eps_ye(rho, eps, ye) / rho;
  }
  AXB_HD double press_from_valid_rho_eps_ye(double rho, double &eps, double ye) const {
    const double lr = lr_clamped(rho);
    const double lt = logtemp(rho, eps, ye);
    return exp(interp(TAB_PRESS, lr, lt, ye));
  }
  // takes the logs of the unclamped inputs, as the reference does (:230-239)
  AXB_HD double press_from_valid_rho_temp_ye(double rho, double temp, double ye) const {
    return exp(interp(TAB_PRESS, log(rho), log(temp), ye));
  }
  AXB_HD double eps_from_valid_rho_temp_ye(double rho, double temp, double ye) const {
    return exp(interp(TAB_EPS, lr_clamped(rho), lt_clamped(temp), ye)) - shift;
  }
  // no inversion of eps(press) for the tabulated EOS: the reference prints a
  // warning, asserts, and with assertions compiled out returns 0
  // (eos_3p_tabulated3d.hxx:259-269); the recovery reaches it only when a
  // limit (v_lim, the table's largest rho, the pressure atmosphere) fires
  // with use_temperature off
  AXB_HD double eps_from_valid_rho_press_ye(double, double, double) const { return 0.0; }
  AXB_HD double csnd_from_valid_rho_eps_ye(double rho, double &eps, double ye) const {
    const double lr = lr_clamped(rho);
    const double lt = logtemp(rho, eps, ye);
    return sqrt(interp(TAB_CS2, lr, lt, ye));
  }
  AXB_HD double temp_from_valid_rho_eps_ye(double rho, double &eps, double ye) const {
    return exp(logtemp(rho, eps, ye));
  }
  AXB_HD double entropy_from_valid_rho_temp_ye(double rho, double temp, double ye) const {
    return interp(TAB_S, lr_clamped(rho), lt_clamped(temp), ye);
  }
  AXB_HD double kappa_from_valid_rho_eps_ye(double rho, double &eps, double ye) const {
    return entropy_from_valid_rho_temp_ye(rho, temp_from_valid_rho_eps_ye(rho, eps, ye), ye);
  }
  // not defined for a table (the reference prints and asserts,
  // eos_3p_tabulated3d.hxx:315-333); the entry points reject the entropy
  // scheme with a tabulated EOS, so these are never reached
  AXB_HD double press_from_valid_rho_kappa_ye(double, double, double) const { return nan(""); }
  AXB_HD double eps_from_valid_rho_kappa_ye(double, double, double) const { return nan(""); }
};

} // namespace axb
