// Test infrastructure only: the subset of CarpetX's Loop library (GF3D2,
// PointDesc, grid loops) that the reference hot-path sources use.
//
// Conventions (CarpetX's): a point index I = (i,j,k) addresses every centring
// of a box with the same strides; cell i lies between vertices i and i+1, so
// face i along a direction is the lower face of cell i.  A box with n interior
// cells and g ghosts stores n+2g cells and n+2g+1 vertices per axis; every grid
// function of the box shares the strides (1, sy, sz).
//
// The loops run over the interior [g, g+n+(vertex?1:0)) per axis, optionally
// widened by ext_c layers in cell-centred and ext_v layers in vertex-centred
// directions.  The widening lets a test evaluate a routine on ghost points
// exactly as a neighbouring box would, which is what the reference's SYNC
// delivers there.  Iterations are independent (each writes only its own point),
// so they are spread over OpenMP threads.
#ifndef AXREF_SHIM_LOOP_DEVICE_HXX
#define AXREF_SHIM_LOOP_DEVICE_HXX

#include <cctk.h>
#include <vec.hxx>

#include <array>

namespace Loop {
using Arith::dim;
using Arith::vect;

template <typename T> struct GF3D2 {
  T *ptr = nullptr;
  long long sy = 0, sz = 0;
  GF3D2() = default;
  GF3D2(T *p, long long sy_, long long sz_) : ptr(p), sy(sy_), sz(sz_) {}
  template <typename U, typename = std::enable_if_t<
                            std::is_same_v<const U, T> && !std::is_same_v<U, T>>>
  GF3D2(const GF3D2<U> &o) : ptr(o.ptr), sy(o.sy), sz(o.sz) {}
  T &operator()(const vect<int, dim> &I) const {
    return ptr[I[0] + sy * I[1] + sz * I[2]];
  }
};

struct PointDesc {
  vect<int, dim> I;
  std::array<vect<int, dim>, dim> DI;
  std::array<CCTK_REAL, dim> DX;
  CCTK_REAL x, y, z;
  int i, j, k;
};

struct GridDescBaseDevice {
  std::array<int, dim> nghostzones;
  std::array<int, dim> ncells;
  std::array<CCTK_REAL, dim> dx;
  std::array<CCTK_REAL, dim> xmin; // coordinate of vertex index g
  int ext_c = 0, ext_v = 0;

  template <int CI, int CJ, int CK, typename F>
  void loop_int_device(const std::array<int, dim> &ng, const F &f) const {
    const int cent[3] = {CI, CJ, CK};
    int lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
      const int e = cent[d] ? ext_c : ext_v;
      lo[d] = ng[d] - e;
      hi[d] = ng[d] + ncells[d] + (cent[d] ? 0 : 1) + e;
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = lo[2]; k < hi[2]; ++k)
      for (int j = lo[1]; j < hi[1]; ++j)
        for (int i = lo[0]; i < hi[0]; ++i) {
          PointDesc p;
          p.I = vect<int, dim>{i, j, k};
          for (int d = 0; d < 3; ++d) {
            p.DI[d] = vect<int, dim>{d == 0, d == 1, d == 2};
            p.DX[d] = dx[d];
          }
          const int idx[3] = {i, j, k};
          CCTK_REAL xyz[3];
          for (int d = 0; d < 3; ++d)
            xyz[d] = xmin[d] + (idx[d] - ng[d] + (cent[d] ? 0.5 : 0.0)) * dx[d];
          p.x = xyz[0];
          p.y = xyz[1];
          p.z = xyz[2];
          p.i = i - ng[0];
          p.j = j - ng[1];
          p.k = k - ng[2];
          f(p);
        }
  }
};

} // namespace Loop

#endif
