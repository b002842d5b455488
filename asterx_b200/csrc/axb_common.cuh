// Common device-side definitions of the B200 engine: box indexing, the
// parameter block, fixed-order tensor contractions and the device error word.
//
// Summation order.  Every contraction adds its terms left to right in index
// order, starting from the first term (the reference's Arith sum<D> starts
// from zero, and 0 + x == x exactly), two-index sums run i outer, j inner.
// Keeping that order is what lets the FP64 results agree with the reference
// to the last bits, up to fused multiply-add contraction.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/asterx_b200.h"

#define AXB_HD __host__ __device__ __forceinline__
#define AXB_D __device__ __forceinline__
#ifdef __CUDACC__
#define AXB_D_ __device__ __forceinline__
#else
#define AXB_D_ inline
#endif

namespace axb {

// Box geometry as the kernels use it.
struct BoxDev {
  int n[3];
  int ng;
  long long sy, sz;
  double dx[3], idx[3];
  double xmin[3];
  // 0: a block covers one row (block x along i, bid.y = j); 1 (batched
  // launches over small boxes): the blocks of a k-plane cover its (i, j)
  // points row after row, so short rows do not leave threads idle
  int packed;

  // the (i, j) of this thread for a range [li, li + ni) x [lj, lj + nj);
  // false outside it
  AXB_D_ bool row_ij(int li, int ni, int lj, int nj, const uint3 bid, int &i, int &j) const {
    if (packed) {
      const int flat = bid.x * blockDim.x + threadIdx.x;
      i = li + flat % ni;
      j = lj + flat / ni;
      return flat < ni * nj;
    }
    i = li + bid.x * blockDim.x + threadIdx.x;
    j = lj + bid.y;
    return i < li + ni;
  }

  AXB_HD long long at(int i, int j, int k) const {
    return (long long)i + sy * j + sz * k;
  }
  AXB_HD long long stride(int d) const { return d == 0 ? 1 : (d == 1 ? sy : sz); }
};

inline BoxDev make_box(const axb_box &b) {
  BoxDev r;
  for (int d = 0; d < 3; ++d) {
    r.n[d] = b.n[d];
    r.dx[d] = b.dx[d];
    r.idx[d] = 1 / b.dx[d];
    r.xmin[d] = b.xmin[d];
  }
  r.ng = b.ng;
  r.sy = b.sy;
  r.sz = b.sz;
  r.packed = 0;
  return r;
}

// 3-vector and symmetric 3x3 matrix helpers in the reference's order.
struct sym3 {
  double xx, xy, xz, yy, yz, zz;
  AXB_HD double operator()(int i, int j) const {
    const int a = i < j ? i : j, b = i < j ? j : i;
    return a == 0 ? (b == 0 ? xx : (b == 1 ? xy : xz))
                  : (a == 1 ? (b == 1 ? yy : yz) : zz);
  }
};

// det by cofactor expansion along the first row (same formula as the
// Arith stand-in used to build the reference checker).
AXB_HD double det3(const sym3 &g) {
  return g.xx * (g.yy * g.zz - g.yz * g.yz) - g.xy * (g.xy * g.zz - g.yz * g.xz) +
         g.xz * (g.xy * g.yz - g.yy * g.xz);
}
AXB_HD sym3 inv3(const sym3 &g, double detg) {
  const double idet = 1 / detg;
  sym3 r;
  r.xx = (g.yy * g.zz - g.yz * g.yz) * idet;
  r.xy = (g.xz * g.yz - g.xy * g.zz) * idet;
  r.xz = (g.xy * g.yz - g.xz * g.yy) * idet;
  r.yy = (g.xx * g.zz - g.xz * g.xz) * idet;
  r.yz = (g.xy * g.xz - g.xx * g.yz) * idet;
  r.zz = (g.xx * g.yy - g.xy * g.xy) * idet;
  return r;
}
// g_ij v^j
AXB_HD void lower3(const sym3 &g, const double v[3], double out[3]) {
  out[0] = g.xx * v[0] + g.xy * v[1] + g.xz * v[2];
  out[1] = g.xy * v[0] + g.yy * v[1] + g.yz * v[2];
  out[2] = g.xz * v[0] + g.yz * v[1] + g.zz * v[2];
}
AXB_HD double dot3(const double a[3], const double b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
AXB_HD double sq(double x) { return x * x; }

// Device error word (AXB_EW_* bits) and the CFL speed accumulator live in a
// small per-context block of device memory.
struct DevStatus {
  unsigned int error_word;
  unsigned int c2p_fail_count;
  unsigned long long max_speed_bits; // non-negative double as ordered bits
  unsigned long long c2p_iter_hist[64];
};

AXB_D void atomic_max_nonneg(unsigned long long *addr, double v) {
  if (!(v >= 0)) return;
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

} // namespace axb
