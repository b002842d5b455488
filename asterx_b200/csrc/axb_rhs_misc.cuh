// Cell, vertex and edge kernels of the RHS group (sources, auxiliaries,
// flux-CT + gauge).  Included by exactly one translation unit.
#pragma once

#include "axb_rhs_kernels.cuh"

namespace axb {

// ---------------------------------------------------------------------------
// k_sources: geometric source terms (AsterX/src/source.cxx:32-167); writes
// the seven hydro RHS (dens, DEnt, DYe sources are zero).
//
// Each vertex field is read once per cell as its 8 cube corners, from which
// the cell average (calc_avg_v2c, AsterUtils/src/aster_interp.hxx) and, at
// second order, the three edge-averaged derivatives (calc_fd_v2c,
// AsterUtils/src/aster_fd.hxx:49-64) are formed in registers.  The
// derivatives multiply by 1/dx once instead of dividing each edge difference
// by dx (last-ulp differences).
// ---------------------------------------------------------------------------
struct V2C {
  double avg, d[3];
};

// corner (bx, by, bz) of the cell at I is c[bx + 2 by + 4 bz]
template <int FD>
AXB_D V2C v2c_field(const double *__restrict__ f, long long I, const BoxDev &b) {
  const long long sy = b.sy, sz = b.sz;
  double c[8];
  c[0] = __ldg(f + I);
  c[1] = __ldg(f + I + 1);
  c[2] = __ldg(f + I + sy);
  c[3] = __ldg(f + I + 1 + sy);
  c[4] = __ldg(f + I + sz);
  c[5] = __ldg(f + I + 1 + sz);
  c[6] = __ldg(f + I + sy + sz);
  c[7] = __ldg(f + I + 1 + sy + sz);
#ifdef AXB_SOURCES_SEQ
  // keep the compiler from hoisting every field's corner loads up front
  asm volatile("" ::: "memory");
#endif
  V2C r;
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q)
    s += c[q];
  r.avg = s / 8.0;
  if (FD == 2) {
    // edges along d from the base corners I, I+s1, I+s2, I+s1+s2
    r.d[0] = ((c[1] - c[0]) + (c[3] - c[2]) + (c[5] - c[4]) + (c[7] - c[6])) * (0.25 * b.idx[0]);
    r.d[1] = ((c[2] - c[0]) + (c[6] - c[4]) + (c[3] - c[1]) + (c[7] - c[5])) * (0.25 * b.idx[1]);
    r.d[2] = ((c[4] - c[0]) + (c[5] - c[1]) + (c[6] - c[2]) + (c[7] - c[3])) * (0.25 * b.idx[2]);
  } else {
    // calc_fd_v2c<4> (aster_fd.hxx:77-110): 4-point differences along each edge
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
      const long long st = b.stride(d), s1 = b.stride(d1), s2 = b.stride(d2);
      const long long base[4] = {I, I + s1, I + s2, I + s1 + s2};
      double e = 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const long long J = base[q];
        e += (1.0 / 24.0) * __ldg(f + J - st) - (27.0 / 24.0) * __ldg(f + J) +
             (27.0 / 24.0) * __ldg(f + J + st) - (1.0 / 24.0) * __ldg(f + J + 2 * st);
      }
      r.d[d] = e * (0.25 * b.idx[d]);
    }
  }
  return r;
}

AXB_D double avg_v2c(const double *__restrict__ f, long long I, long long sy,
                     long long sz) {
  double s = 0.0;
  s += __ldg(f + I);
  s += __ldg(f + I + 1);
  s += __ldg(f + I + sy);
  s += __ldg(f + I + 1 + sy);
  s += __ldg(f + I + sz);
  s += __ldg(f + I + 1 + sz);
  s += __ldg(f + I + sy + sz);
  s += __ldg(f + I + 1 + sy + sz);
  return s / 8.0;
}

AXB_HD double sym_get(const sym3 &m, int p, int q) { return m(p, q); }

#ifndef AXB_SOURCES_SMEM
#define AXB_SOURCES_SMEM 1
#endif
#ifndef AXB_SOURCES_MINB
#define AXB_SOURCES_MINB 3
#endif
template <int FD>
AXB_D void sources_cell(const RhsArgs &a, const int i, const int j, const int k) {
  const BoxDev &b = a.b;
  const long long I = b.at(i, j, k);
  const long long sy = b.sy, sz = b.sz;
#if AXB_SOURCES_SMEM
  // the 30 metric derivatives wait in shared memory (one column per thread)
  // until the stress tensor is formed: in registers they pushed the kernel
  // to 255 registers and 8 warps per SM
  __shared__ double s_der[30][128];
  const int tl = threadIdx.x;
#define AXB_DALP(d) s_der[(d)][tl]
#define AXB_DBETA(d, q) s_der[3 + 3 * (d) + (q)][tl]
#define AXB_DG(d, q) s_der[12 + 6 * (d) + (q)][tl]
#else
  double d_alp_r[3], d_beta_r[3][3], d_g_r[3][6];
#define AXB_DALP(d) d_alp_r[d]
#define AXB_DBETA(d, q) d_beta_r[d][q]
#define AXB_DG(d, q) d_g_r[d][q]
#endif
  double alp, beta[3];
  sym3 g, K;
  {
    const V2C r = v2c_field<FD>(a.alp, I, b);
    alp = r.avg;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      AXB_DALP(d) = r.d[d];
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const V2C r = v2c_field<FD>(a.beta[q], I, b);
    beta[q] = r.avg;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      AXB_DBETA(d, q) = r.d[d];
  }
  double gv[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const V2C r = v2c_field<FD>(a.g[q], I, b);
    gv[q] = r.avg;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      AXB_DG(d, q) = r.d[d];
  }
  g = sym3{gv[0], gv[1], gv[2], gv[3], gv[4], gv[5]};
  K.xx = avg_v2c(a.K[0], I, sy, sz);
  K.xy = avg_v2c(a.K[1], I, sy, sz);
  K.xz = avg_v2c(a.K[2], I, sy, sz);
  K.yy = avg_v2c(a.K[3], I, sy, sz);
  K.yz = avg_v2c(a.K[4], I, sy, sz);
  K.zz = avg_v2c(a.K[5], I, sy, sz);
  const double detg = det3(g);
  const double sqrt_detg = sqrt(detg);
  const sym3 ug = inv3(g, detg);
  const double v_up[3] = {a.vel[0][I], a.vel[1][I], a.vel[2][I]};
  double v_low[3];
  lower3(g, v_up, v_low);
  const double w = 1.0 / sqrt(1.0 - dot3(v_low, v_up));
  const double rho = a.rho[I], eps = a.eps[I], press = a.press[I];
  const double rhW2 = (rho * (1.0 + eps) + press) * w * w;
  const double ialp = 1.0 / alp;
  double vs[3];
#pragma unroll
  for (int q = 0; q < 3; ++q)
    vs[q] = v_up[q] - beta[q] * ialp;
  const double B_up[3] = {a.Bvec[0][I], a.Bvec[1][I], a.Bvec[2][I]};
  double B_low[3];
  lower3(g, B_up, B_low);
  const double bs0 = w * dot3(B_up, v_low) * ialp;
  double bs[3];
#pragma unroll
  for (int q = 0; q < 3; ++q)
    bs[q] = B_up[q] / w + alp * bs0 * vs[q];
  const double bs2 = (dot3(B_up, B_low) + sq(alp * bs0)) / sq(w);
  double gb[3], gbs[3], bs_low[3];
  lower3(g, beta, gb);
  lower3(g, bs, gbs);
#pragma unroll
  for (int q = 0; q < 3; ++q)
    bs_low[q] = gb[q] * bs0 + gbs[q];
  const double A = rhW2 + bs2 * sq(w);
  const double P = press + 0.5 * bs2;
  const double ialp2 = 1.0 / sq(alp);
  const double t00 = (A - P) * ialp2 - sq(bs0);
  double t0[3], t0low[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    t0[q] = A * vs[q] * ialp + P * beta[q] * ialp2 - bs0 * bs[q];
    t0low[q] = A * v_low[q] * ialp - bs_low[q] * bs0;
  }
  // T^{ij} is symmetric (an smat in the reference): upper triangle, mirrored
  double t[3][3];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = p; q < 3; ++q)
      t[p][q] = t[q][p] = A * vs[p] * vs[q] +
                          P * (ug(p, q) - beta[p] * beta[q] * ialp2) - bs[p] * bs[q];
  double shiftk[3];
  lower3(K, beta, shiftk);
  const double ssk = dot3(shiftk, beta);
  double X[3];
#pragma unroll
  for (int q = 0; q < 3; ++q)
    X[q] = -AXB_DALP(q) + 2.0 * shiftk[q];
  double Kt = 0.0;
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q)
      Kt += K(p, q) * t[p][q];
  const double d_alp3[3] = {AXB_DALP(0), AXB_DALP(1), AXB_DALP(2)};
  const double tau_source = t00 * (ssk - dot3(beta, d_alp3)) + dot3(t0, X) + Kt;
  double ms[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const sym3 dgd{AXB_DG(d, 0), AXB_DG(d, 1), AXB_DG(d, 2),
                   AXB_DG(d, 3), AXB_DG(d, 4), AXB_DG(d, 5)};
    double nrm = 0.0, c1 = 0.0, c3 = 0.0;
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const double dg = dgd(p, q);
        nrm += dg * beta[p] * beta[q];
        c1 += dg * t0[p] * beta[q];
        c3 += t[p][q] * dg;
      }
    const double dbd[3] = {AXB_DBETA(d, 0), AXB_DBETA(d, 1), AXB_DBETA(d, 2)};
    const double c2 = dot3(t0low, dbd);
    ms[d] = t00 * (0.5 * nrm - alp * AXB_DALP(d)) + c1 + c2 + 0.5 * c3;
  }
#undef AXB_DALP
#undef AXB_DBETA
#undef AXB_DG
  const double as = alp * sqrt_detg;
  a.rhs[V_DENS][I] = 0.0;
  a.rhs[V_DENT][I] = 0.0;
  a.rhs[V_MOMX][I] = as * ms[0];
  a.rhs[V_MOMY][I] = as * ms[1];
  a.rhs[V_MOMZ][I] = as * ms[2];
  a.rhs[V_TAU][I] = as * tau_source;
  a.rhs[V_DYE][I] = 0.0;
}
template <int FD>
AXB_D void sources_body(const RhsArgs &a, const uint3 bid) {
  int i, j;
  const int k = a.b.ng + bid.z;
  if (!a.b.row_ij(a.b.ng, a.b.n[0], a.b.ng, a.b.n[1], bid, i, j))
    return;
  sources_cell<FD>(a, i, j, k);
}

// A thread walks `seg` cells up a z column (block z = segment), prefetching
// into L2 the rows the next cell adds: the upper vertex plane of the 16
// metric fields and the cell's primitives (its lower vertex plane is the
// current cell's upper one).
#ifndef AXB_SOURCES_SEG
#define AXB_SOURCES_SEG 16 // cells per thread along z; 0 or 1: one cell
#endif
template <int FD>
AXB_D void sources_column(const RhsArgs &a, const uint3 bid, const int seg) {
  const BoxDev &b = a.b;
  int i, j;
  if (!b.row_ij(b.ng, b.n[0], b.ng, b.n[1], bid, i, j))
    return;
  const int k0 = b.ng + int(bid.z) * seg;
  const int k1 = min(k0 + seg, b.ng + b.n[2]);
  for (int k = k0; k < k1; ++k) {
    if (k + 1 < k1) {
      const long long J = b.at(i, j, k + 2); // upper vertex plane of cell k+1
      const long long C = b.at(i, j, k + 1);
      const long long sy = b.sy;
      prefetch_l2(a.alp + J);
      prefetch_l2(a.alp + J + sy);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        prefetch_l2(a.beta[q] + J);
        prefetch_l2(a.beta[q] + J + sy);
      }
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        prefetch_l2(a.g[q] + J);
        prefetch_l2(a.g[q] + J + sy);
        prefetch_l2(a.K[q] + J);
        prefetch_l2(a.K[q] + J + sy);
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        prefetch_l2(a.vel[q] + C);
        prefetch_l2(a.Bvec[q] + C);
      }
      prefetch_l2(a.rho + C);
      prefetch_l2(a.eps + C);
      prefetch_l2(a.press + C);
    }
    sources_cell<FD>(a, i, j, k);
  }
}

template <int FD>
__global__ void __launch_bounds__(128, AXB_SOURCES_MINB)
    k_sources(const RhsArgs a) {
  sources_body<FD>(a, blockIdx);
}
template <int FD>
__global__ void __launch_bounds__(128, AXB_SOURCES_MINB)
    k_sources_column(const RhsArgs a, const int seg) {
  sources_column<FD>(a, blockIdx, seg);
}

// ---------------------------------------------------------------------------
// k_aux: vertex auxiliaries of the A/Psi RHS (fluxes.cxx:798-826) on the
// vertices [ng-2, ng+n+2] (the Psi RHS reads F at +-1 and Fbeta at +-2).
// ---------------------------------------------------------------------------
AXB_D void aux_body(const RhsArgs &a, const uint3 bid) {
  const BoxDev &b = a.b;
  int i, j;
  const int k = b.ng - 2 + bid.z;
  if (!b.row_ij(b.ng - 2, b.n[0] + 5, b.ng - 2, b.n[1] + 5, bid, i, j))
    return;
  const long long I = b.at(i, j, k);
  double Av[3];
  for (int d = 0; d < 3; ++d) {
    double s = 0.0;
    s += a.Avec[d][I];
    s += a.Avec[d][I - b.stride(d)];
    Av[d] = s / 2.0;
  }
  const sym3 g{a.g[0][I], a.g[1][I], a.g[2][I], a.g[3][I], a.g[4][I], a.g[5][I]};
  const double be[3] = {a.beta[0][I], a.beta[1][I], a.beta[2][I]};
  const double detg = det3(g);
  const double sqrtg = sqrt(detg);
  const sym3 ug = inv3(g, detg);
  double Aup[3];
  lower3(ug, Av, Aup);
  const double alp = a.alp[I], psi = a.Psi[I];
  a.aux[0][I] = alp * sqrtg * Aup[0];
  a.aux[1][I] = alp * sqrtg * Aup[1];
  a.aux[2][I] = alp * sqrtg * Aup[2];
  a.aux[3][I] = be[0] * psi;
  a.aux[4][I] = be[1] * psi;
  a.aux[5][I] = be[2] * psi;
  a.aux[6][I] = alp * psi / sqrtg - dot3(be, Av);
}
__global__ void __launch_bounds__(128)
    k_aux(const RhsArgs a) {
  aux_body(a, blockIdx);
}

// ---------------------------------------------------------------------------
// k_ct_psi: on every interior vertex (i,j,k): the x-, y-, z-edge starting
// there (when it is interior) gets Avec_rhs = -E - dG (flux-CT E from the
// stored face B fluxes, rhs.cxx:171-185), and the vertex gets Psi_rhs
// (rhs.cxx:227-252).
// ---------------------------------------------------------------------------
// Upwind-CT edge electric field (AsterX_RHS with use_uct, rhs.cxx:124-168)
// of the e-edge at I: the staggered B and the upwind-averaged vtilde of the
// two adjacent face sets, reconstructed to the edge along the other
// transverse direction (ReconX reconstruct with the cell-centred press and
// velocity, not rho), weighted by the bounding speeds of the faces.
template <int RECON>
AXB_D double uct_edge_E(const RhsArgs &a, long long I, int e) {
  const BoxDev &b = a.b;
  const int ej = (e + 1) % 3, ek = (e + 2) % 3;
  // the interface values at I along d: upper value of the cell at I - s
  // (left) and lower value of the cell at I (right)
  auto rc = [&](const double *f, int d, double &L, double &R) {
    const long long s = b.stride(d);
    double q[5], pr[5], vd[5];
    load_pencil<5>(f, I - s, s, q);
    load_pencil<5>(a.press, I - s, s, pr);
    load_pencil<5>(a.vel[d], I - s, s, vd);
    L = recon_cell<RECON>(q, pr, vd, false, a.rp).up;
    load_pencil<5>(f, I, s, q);
    load_pencil<5>(a.press, I, s, pr);
    load_pencil<5>(a.vel[d], I, s, vd);
    R = recon_cell<RECON>(q, pr, vd, false, a.rp).lo;
  };
  // one: B and vtilde^{ek} on the ej-faces, along ek, speeds of the ek-face
  double B1L, B1R, v1L, v1R;
  rc(a.dBstag[ej], ek, B1L, B1R);
  rc(a.uct[4 * ej + 0], ek, v1L, v1R);
  const double amax1 = a.uct[4 * ek + 2][I], amin1 = a.uct[4 * ek + 3][I];
  // two: B and vtilde^{ej} on the ek-faces, along ej, speeds of the ej-face
  double B2L, B2R, v2L, v2R;
  rc(a.dBstag[ek], ej, B2L, B2R);
  rc(a.uct[4 * ek + 1], ej, v2L, v2R);
  const double amax2 = a.uct[4 * ej + 2][I], amin2 = a.uct[4 * ej + 3][I];
  double E = (amax1 * v1L * B1L + amin1 * v1R * B1R - amax1 * amin1 * (B1R - B1L)) /
             (amax1 + amin1);
  E -= (amax2 * v2L * B2L + amin2 * v2R * B2R - amax2 * amin2 * (B2R - B2L)) /
       (amax2 + amin2);
  return E;
}

// UCT_RECON < 0: flux-CT edge field; otherwise upwind CT with that
// reconstruction.
template <int UCT_RECON>
AXB_D void ct_psi_body(const RhsArgs &a, const uint3 bid) {
  const BoxDev &b = a.b;
  const int ng = b.ng;
  int i, j;
  const int k = ng + bid.z;
  if (!b.row_ij(ng, b.n[0] + 1, ng, b.n[1] + 1, bid, i, j))
    return;
  const long long I = b.at(i, j, k);
  const int ijk[3] = {i, j, k};
  const bool gl = a.gauge == AXB_GAUGE_GEN_LORENZ;
  const double *G = a.aux[6];
  // bflux: 0 fxBy 1 fxBz 2 fyBx 3 fyBz 4 fzBx 5 fzBy
  for (int e = 0; e < 3; ++e) {
    if (ijk[e] >= ng + b.n[e])
      continue;
    double E;
    if constexpr (UCT_RECON >= 0) {
      E = uct_edge_E<UCT_RECON>(a, I, e);
    } else {
      const int ej = (e + 1) % 3, ek = (e + 2) % 3;
      // fBs(j)(k): flux along k of B_j; fBs(k)(j): flux along j of B_k
      const double *fjk, *fkj;
      if (e == 0) {
        fjk = a.bflux[5]; // fzBy
        fkj = a.bflux[3]; // fyBz
      } else if (e == 1) {
        fjk = a.bflux[1]; // fxBz
        fkj = a.bflux[4]; // fzBx
      } else {
        fjk = a.bflux[2]; // fyBx
        fkj = a.bflux[0]; // fxBy
      }
      E = 0.25 * ((fjk[I] + fjk[I - b.stride(ej)]) - (fkj[I] + fkj[I - b.stride(ek)]));
    }
    double r = -E;
    if (gl)
      r = -E - (G[I + b.stride(e)] - G[I]) / b.dx[e];
    if (a.fuse_stage)
      a.st_uk[7 + e][I] = stage_combine(a.st_alpha, a.st_un[7 + e][I], a.st_beta,
                                        a.st_uk[7 + e][I], a.st_gdt, r);
    else
      a.Arhs[e][I] = r;
  }
  if (gl) {
    double dF = 0.0;
    for (int d = 0; d < 3; ++d) {
      const long long s = b.stride(d);
      const double *F = a.aux[d], *Fb = a.aux[3 + d];
      const double c2c = (0.5 / b.dx[d]) * (F[I + s] - F[I - s]);
      const int sg = a.beta[d][I] < 0 ? -1 : 1;
      const double one =
          -sg * (Fb[I + 2 * sg * s] - 4.0 * Fb[I + sg * s] + 3.0 * Fb[I]) *
          (0.5 / b.dx[d]);
      dF += c2c - one;
    }
    const double r = -dF - a.lorenz_damp_fac * a.alp[I] * a.Psi[I];
    if (a.fuse_stage) // Psi is read above at this vertex only
      a.st_uk[10][I] = stage_combine(a.st_alpha, a.st_un[10][I], a.st_beta,
                                     a.st_uk[10][I], a.st_gdt, r);
    else
      a.Psi_rhs[I] = r;
  } else {
    if (a.fuse_stage)
      a.st_uk[10][I] = stage_combine(a.st_alpha, a.st_un[10][I], a.st_beta,
                                     a.st_uk[10][I], a.st_gdt, 0.0);
    else
      a.Psi_rhs[I] = 0.0;
  }
}
__global__ void __launch_bounds__(128)
    k_ct_psi(const RhsArgs a) {
  ct_psi_body<-1>(a, blockIdx);
}
template <int RECON>
__global__ void __launch_bounds__(128)
    k_ct_psi_uct(const RhsArgs a) {
  ct_psi_body<RECON>(a, blockIdx);
}

} // namespace axb
