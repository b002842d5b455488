// Test infrastructure only: stand-in for CarpetX's Algo::brent (external,
// unvendored: scripts/asterx.th:698-700).  Its contract is taken from the
// reference call site Con2PrimFactory/src/c2p_1DPalenzuela.hxx:380-417:
//   brent(f, a, b, minbits, maxiters, iters) -> pair (lo, hi)
// returns a bracket of a sign change of f and stops once
//   |hi - lo| <= 2^-minbits * min(|lo|, |hi|)
// or after maxiters iterations; iters receives the iteration count.
//
// The body is Brent's method (R. P. Brent, "Algorithms for Minimization
// without Derivatives", 1973) in its common inverse-quadratic / secant /
// bisection form: the iterate b is the best estimate, a the contrapoint, so
// [a, b] always brackets the root.  The oracle restatement and the CUDA
// kernels implement the same steps (axo::brent_bracket, axb brent_bracket).
#ifndef AXREF_SHIM_ROOTS_HXX
#define AXREF_SHIM_ROOTS_HXX

#include <cctk.h>

#include <algorithm>
#include <cmath>
#include <utility>

namespace Algo {

template <typename F, typename T>
std::pair<T, T> brent(const F &f, T a, T b, const int minbits,
                      const int maxiters, int &iters) {
  using std::fabs;
  const T eps = std::ldexp(T(1), -minbits);
  T fa = f(a);
  T fb = f(b);
  iters = 0;
  if (fa == 0)
    return {a, a};
  if (fb == 0)
    return {b, b};
  if (fa * fb > 0) // not bracketed: hand the interval back unchanged
    return {std::min(a, b), std::max(a, b)};
  if (fabs(fa) < fabs(fb)) {
    std::swap(a, b);
    std::swap(fa, fb);
  }
  T c = a, fc = fa, d = a;
  bool mflag = true;
  while (iters < maxiters) {
    if (fabs(b - a) <= eps * std::min(fabs(a), fabs(b)))
      break;
    ++iters;
    T s;
    if (fa != fc && fb != fc) {
      s = a * fb * fc / ((fa - fb) * (fa - fc)) +
          b * fa * fc / ((fb - fa) * (fb - fc)) +
          c * fa * fb / ((fc - fa) * (fc - fb));
    } else {
      s = b - fb * (b - a) / (fb - fa);
    }
    const T delta = eps * fabs(b);
    const T q = (3 * a + b) / 4;
    const bool out_of_range = !((s > std::min(q, b)) && (s < std::max(q, b)));
    if (out_of_range || (mflag && fabs(s - b) >= fabs(b - c) / 2) ||
        (!mflag && fabs(s - b) >= fabs(c - d) / 2) ||
        (mflag && fabs(b - c) < delta) || (!mflag && fabs(c - d) < delta)) {
      s = (a + b) / 2;
      mflag = true;
    } else {
      mflag = false;
    }
    const T fs = f(s);
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
      std::swap(a, b);
      std::swap(fa, fb);
    }
    if (fb == 0)
      return {b, b};
  }
  return {std::min(a, b), std::max(a, b)};
}

} // namespace Algo

#endif
