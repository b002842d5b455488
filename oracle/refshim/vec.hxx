// Test infrastructure only: the subset of CarpetX's Arith library (vec, vect,
// smat, sum, pow2, calc_det, calc_inv) that the reference hot-path headers
// use, written here from the mathematics so the reference sources compile
// unmodified on the host.  CarpetX is an external, unvendored dependency of
// the reference (scripts/asterx.th:698-700, default branch, no pinned
// revision); its call sites are AsterX/src/fluxes.cxx:235,659,
// AsterX/src/source.cxx:47-50, Con2PrimFactory/src/c2p.hxx:278-279,338-341,
// Con2PrimFactory/src/c2p_2DNoble.hxx:288,310.
//
// Summation order is fixed and documented here because it decides the last
// bits of every contraction: sum<D>(f) adds f(0), f(1), ... left to right
// starting from zero; the two-index forms run i outer, j inner.  The oracle
// restatement and the CUDA kernels follow the same order.
#ifndef AXREF_SHIM_VEC_HXX
#define AXREF_SHIM_VEC_HXX

#include <cctk.h>

#include <array>
#include <cassert>
#include <cmath>
#include <initializer_list>
#include <type_traits>
#include <utility>

namespace Arith {

constexpr int dim = 3;

template <typename T> constexpr inline T pow2(const T &x) { return x * x; }

template <typename T, int N> struct vect;
template <typename T, int N> struct vec;

namespace detail {
template <typename X> struct is_vecish : std::false_type {};
template <typename T, int N> struct is_vecish<vec<T, N>> : std::true_type {};
template <typename T, int N> struct is_vecish<vect<T, N>> : std::true_type {};
template <typename T, std::size_t N>
struct is_vecish<std::array<T, N>> : std::true_type {};
} // namespace detail

// Small fixed-size vector with element-wise arithmetic.
template <typename T, int N> struct vec {
  std::array<T, N> elts;

  vec() = default;
  vec(const vec &) = default;
  vec &operator=(const vec &) = default;
  vec(std::initializer_list<T> l) {
    assert(int(l.size()) == N);
    int i = 0;
    for (const auto &x : l)
      elts[i++] = x;
  }
  vec(const std::array<T, N> &a) : elts(a) {}
  template <typename U, typename = std::enable_if_t<!std::is_same_v<U, T>>>
  vec(const vec<U, N> &o) {
    for (int i = 0; i < N; ++i)
      elts[i] = T(o.elts[i]);
  }
  template <typename F,
            typename = std::enable_if_t<
                !detail::is_vecish<std::decay_t<F>>::value &&
                std::is_invocable_v<const F &, int>>>
  vec(const F &f) {
    for (int i = 0; i < N; ++i)
      elts[i] = f(i);
  }

  static vec unit(int d) {
    vec r;
    for (int i = 0; i < N; ++i)
      r.elts[i] = T(i == d);
    return r;
  }

  T &operator()(int i) { return elts[i]; }
  const T &operator()(int i) const { return elts[i]; }
  T &operator[](int i) { return elts[i]; }
  const T &operator[](int i) const { return elts[i]; }

  vec &operator+=(const vec &o) {
    for (int i = 0; i < N; ++i)
      elts[i] += o.elts[i];
    return *this;
  }
  vec &operator-=(const vec &o) {
    for (int i = 0; i < N; ++i)
      elts[i] -= o.elts[i];
    return *this;
  }
  template <typename S> vec &operator*=(const S &s) {
    for (int i = 0; i < N; ++i)
      elts[i] *= s;
    return *this;
  }
  template <typename S> vec &operator/=(const S &s) {
    for (int i = 0; i < N; ++i)
      elts[i] /= s;
    return *this;
  }
};

template <typename T, int N> vec<T, N> operator+(const vec<T, N> &a) {
  return a;
}
template <typename T, int N> vec<T, N> operator-(const vec<T, N> &a) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i)
    r.elts[i] = -a.elts[i];
  return r;
}
template <typename T, int N>
vec<T, N> operator+(const vec<T, N> &a, const vec<T, N> &b) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i)
    r.elts[i] = a.elts[i] + b.elts[i];
  return r;
}
template <typename T, int N>
vec<T, N> operator-(const vec<T, N> &a, const vec<T, N> &b) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i)
    r.elts[i] = a.elts[i] - b.elts[i];
  return r;
}
template <typename T, int N>
vec<T, N> operator*(const T &s, const vec<T, N> &a) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i)
    r.elts[i] = s * a.elts[i];
  return r;
}
template <typename T, int N>
vec<T, N> operator*(const vec<T, N> &a, const T &s) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i)
    r.elts[i] = a.elts[i] * s;
  return r;
}
template <typename T, int N>
vec<T, N> operator/(const vec<T, N> &a, const T &s) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i)
    r.elts[i] = a.elts[i] / s;
  return r;
}

// Integer index vector (grid point indices and offsets).
template <typename T, int N> struct vect {
  std::array<T, N> elts;
  vect() = default;
  vect(std::initializer_list<T> l) {
    assert(int(l.size()) == N);
    int i = 0;
    for (const auto &x : l)
      elts[i++] = x;
  }
  T &operator[](int i) { return elts[i]; }
  const T &operator[](int i) const { return elts[i]; }
  T &operator()(int i) { return elts[i]; }
  const T &operator()(int i) const { return elts[i]; }
};
template <typename T, int N>
vect<T, N> operator+(const vect<T, N> &a, const vect<T, N> &b) {
  vect<T, N> r;
  for (int i = 0; i < N; ++i)
    r.elts[i] = a.elts[i] + b.elts[i];
  return r;
}
template <typename T, int N>
vect<T, N> operator-(const vect<T, N> &a, const vect<T, N> &b) {
  vect<T, N> r;
  for (int i = 0; i < N; ++i)
    r.elts[i] = a.elts[i] - b.elts[i];
  return r;
}
template <typename T, int N> vect<T, N> operator*(const T &s, const vect<T, N> &a) {
  vect<T, N> r;
  for (int i = 0; i < N; ++i)
    r.elts[i] = s * a.elts[i];
  return r;
}
template <typename T, int N> vect<T, N> operator*(const vect<T, N> &a, const T &s) {
  vect<T, N> r;
  for (int i = 0; i < N; ++i)
    r.elts[i] = a.elts[i] * s;
  return r;
}

// Symmetric matrix, stored xx, xy, xz, yy, yz, zz.
template <typename T, int D> struct smat;
template <typename T> struct smat<T, 3> {
  std::array<T, 6> elts;
  static constexpr int ind(int i, int j) {
    return i <= j ? (i == 0 ? j : (i == 1 ? 2 + j : 5))
                  : (j == 0 ? i : (j == 1 ? 2 + i : 5));
  }
  smat() = default;
  smat(std::initializer_list<T> l) {
    assert(l.size() == 6);
    int i = 0;
    for (const auto &x : l)
      elts[i++] = x;
  }
  template <typename F, typename = std::enable_if_t<
                            std::is_invocable_v<const F &, int, int>>>
  smat(const F &f) {
    for (int i = 0; i < 3; ++i)
      for (int j = i; j < 3; ++j)
        elts[ind(i, j)] = f(i, j);
  }
  T &operator()(int i, int j) { return elts[ind(i, j)]; }
  const T &operator()(int i, int j) const { return elts[ind(i, j)]; }
};

// Sums in a fixed order: index 0 first, accumulator starts at zero.
template <int D, typename F> inline auto sum(const F &f) {
  if constexpr (std::is_invocable_v<const F &, int>) {
    using R = std::decay_t<decltype(f(0))>;
    R s = 0;
    for (int i = 0; i < D; ++i)
      s += f(i);
    return s;
  } else {
    using R = std::decay_t<decltype(f(0, 0))>;
    R s = 0;
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j)
        s += f(i, j);
    return s;
  }
}
// Full double sum over a symmetric pair of indices (i outer, j inner).
template <int D, typename F> inline auto sum_symm(const F &f) {
  using R = std::decay_t<decltype(f(0, 0))>;
  R s = 0;
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j)
      s += f(i, j);
  return s;
}

// Determinant of a symmetric 3x3 matrix by cofactor expansion along the
// first row.
template <typename T> inline T calc_det(const smat<T, 3> &g) {
  return g(0, 0) * (g(1, 1) * g(2, 2) - g(1, 2) * g(1, 2)) -
         g(0, 1) * (g(0, 1) * g(2, 2) - g(1, 2) * g(0, 2)) +
         g(0, 2) * (g(0, 1) * g(1, 2) - g(1, 1) * g(0, 2));
}
// Inverse of a symmetric 3x3 matrix from its adjugate and determinant.
template <typename T> inline smat<T, 3> calc_inv(const smat<T, 3> &g, const T &detg) {
  const T idet = 1 / detg;
  smat<T, 3> r;
  r(0, 0) = (g(1, 1) * g(2, 2) - g(1, 2) * g(1, 2)) * idet;
  r(0, 1) = (g(0, 2) * g(1, 2) - g(0, 1) * g(2, 2)) * idet;
  r(0, 2) = (g(0, 1) * g(1, 2) - g(0, 2) * g(1, 1)) * idet;
  r(1, 1) = (g(0, 0) * g(2, 2) - g(0, 2) * g(0, 2)) * idet;
  r(1, 2) = (g(0, 1) * g(0, 2) - g(0, 0) * g(1, 2)) * idet;
  r(2, 2) = (g(0, 0) * g(1, 1) - g(0, 1) * g(0, 1)) * idet;
  return r;
}

} // namespace Arith

#endif
