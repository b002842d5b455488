// RHS kernels (see axb_rhs.cuh for the overview).
#pragma once

#include "axb_rhs.cuh"

namespace axb {

template <int N>
AXB_D void load_pencil(const double *__restrict__ f, long long I, long long s,
                       double (&q)[N]) {
#pragma unroll
  for (int m = 0; m < N; ++m)
    q[m] = __ldg(f + I + (m - N / 2) * s);
}

AXB_D double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---------------------------------------------------------------------------
// k_flux_pass: one thread marches one pencil segment along DIR.  Per step it
// reconstructs one cell (both interface values, ReconX per-cell formulas),
// forms the face between the previous cell and this one, computes the ten
// Riemann fluxes, stores the two transverse B fluxes (for flux-CT), and
// folds F(face) - F(face-1) into the partial divergence of the previous cell.
// Threads of a warp are adjacent along the fast transverse axis, so every
// load of a y- or z-pass is a coalesced 256-byte row.
// Transverse range: cells [ng-1, ng+n] (one ghost layer each side, needed
// by the edge electric field); faces along DIR: [ng, ng+n].
// ---------------------------------------------------------------------------
template <int DIR, int RECON, class EOS>
__global__ void __launch_bounds__(128)
    k_flux_pass(const RhsArgs a, const EOS eos, const int seglen) {
  constexpr int D1 = (DIR + 1) % 3, D2 = (DIR + 2) % 3;
  constexpr int T0 = (DIR == 0) ? 1 : 0;
  constexpr int T1 = (DIR == 2) ? 1 : 2;
  const BoxDev &b = a.b;
  const int ng = b.ng;
  const int t0 = ng - 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int t1 = ng - 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const bool active = (t0 <= ng + b.n[T0]) && (t1 <= ng + b.n[T1]);
  double smax = 0.0;
  bool bad = false;
  if (active) {
    const bool trans_int = (t0 >= ng) && (t0 < ng + b.n[T0]) && (t1 >= ng) &&
                           (t1 < ng + b.n[T1]);
    const int f0 = ng + blockIdx.z * seglen;
    const int flast = min(f0 + seglen, ng + b.n[DIR]);
    const long long sd = b.stride(DIR);
    int ijk[3];
    ijk[T0] = t0;
    ijk[T1] = t1;
    ijk[DIR] = f0 - 1;
    long long I = b.at(ijk[0], ijk[1], ijk[2]);
    const double *fld[NREC] = {a.rho,    a.entropy, a.Ye,       a.thermo,
                               a.vel[0], a.vel[1],  a.vel[2],   a.Bvec[D1],
                               a.Bvec[D2]};
    const double idxd = b.idx[DIR];
    double upL[NREC];
    double Fprev[NHYDRO];
    for (int c = f0 - 1; c <= flast; ++c, I += sd) {
      double lo[NREC], up[NREC];
      double pr[5], vd[5];
      load_pencil<5>(a.press, I, sd, pr);
      load_pencil<5>(a.vel[DIR], I, sd, vd);
#pragma unroll
      for (int v = 0; v < NREC; ++v) {
        double q[5];
        if (v == R_PRESS && !a.rec_temp) {
#pragma unroll
          for (int m = 0; m < 5; ++m) q[m] = pr[m];
        } else if (v == R_VX + DIR) {
#pragma unroll
          for (int m = 0; m < 5; ++m) q[m] = vd[m];
        } else {
          load_pencil<5>(fld[v], I, sd, q);
        }
        const CellLoUp r = recon_cell<RECON>(q, pr, vd, v == R_RHO, a.rp);
        lo[v] = r.lo;
        up[v] = r.up;
      }
      if (c >= f0) {
        // face c: left state = upper values of cell c-1, right = lower of c
        double L[NREC], R[NREC];
#pragma unroll
        for (int v = 0; v < NREC; ++v) {
          L[v] = upL[v];
          R[v] = lo[v];
        }
        const bool lo0 = (L[R_RHO] <= 0.0) || (L[R_ENT] <= 0.0) ||
                         (L[R_YE] <= 0.0) || (L[R_PRESS] <= 0.0);
        const bool lo1 = (R[R_RHO] <= 0.0) || (R[R_ENT] <= 0.0) ||
                         (R[R_YE] <= 0.0) || (R[R_PRESS] <= 0.0);
        if (lo0 || lo1) { // low-order redo (fluxes.cxx:313-343)
          for (int v = 0; v < NREC; ++v) {
            double q[5];
            if (lo0) {
              load_pencil<5>(fld[v], I - sd, sd, q);
              L[v] = recon_cell_lo(a.recon_lo, q).up;
            }
            if (lo1) {
              load_pencil<5>(fld[v], I, sd, q);
              R[v] = recon_cell_lo(a.recon_lo, q).lo;
            }
          }
        }
        const FaceMetric m = face_metric<DIR>(a, I);
        const double Bdir = __ldg(a.dBstag[DIR] + I) / m.sqrtg;
        SideOut sL, sR;
        side_physics<DIR>(m, L, Bdir, eos, a.rec_temp, sL);
        side_physics<DIR>(m, R, Bdir, eos, a.rec_temp, sR);
        const double cmax = fmax(0.0, fmax(fmax(sL.lam_p, sL.lam_m),
                                           fmax(sR.lam_p, sR.lam_m)));
        const double cmin = fmin(0.0, fmin(fmin(sL.lam_p, sL.lam_m),
                                           fmin(sR.lam_p, sR.lam_m)));
        smax = fmax(smax, fmax(cmax, -cmin));
        double F[10];
        if (a.flux_type == AXB_FLUX_HLLE) {
          const double cpm = cmax - cmin;
#pragma unroll
          for (int v = 0; v < 10; ++v)
            F[v] = (cmax * sL.F[v] - cmin * sR.F[v] +
                    cmax * cmin * (sR.U[v] - sL.U[v])) /
                   cpm;
        } else {
          const double ch = fmax(cmax, -cmin);
#pragma unroll
          for (int v = 0; v < 10; ++v)
            F[v] = 0.5 * ((sL.F[v] + sR.F[v]) - ch * (sR.U[v] - sL.U[v]));
        }
#pragma unroll
        for (int v = 0; v < 10; ++v)
          bad |= isnan(F[v]);
        if (a.write_bflux) {
          // bflux slots per direction hold the two transverse components in
          // ascending order: x (y, z), y (x, z), z (x, y)
          constexpr int BLO = D1 < D2 ? D1 : D2, BHI = D1 < D2 ? D2 : D1;
          a.bflux[2 * DIR + 0][I] = F[7 + BLO];
          a.bflux[2 * DIR + 1][I] = F[7 + BHI];
        }
        if (c > f0 && trans_int) {
          const long long Ic = I - sd;
#pragma unroll
          for (int v = 0; v < NHYDRO; ++v) {
            const double dF = F[v] - Fprev[v];
            if (DIR == 0)
              a.acc[v][Ic] = idxd * dF;
            else if (DIR == 1)
              a.acc[v][Ic] = a.acc[v][Ic] + idxd * dF;
            else
              a.rhs[v][Ic] = a.rhs[v][Ic] + (-(a.acc[v][Ic] + idxd * dF));
          }
        }
#pragma unroll
        for (int v = 0; v < NHYDRO; ++v)
          Fprev[v] = F[v];
      }
#pragma unroll
      for (int v = 0; v < NREC; ++v)
        upL[v] = up[v];
    }
  }
  // characteristic-speed maximum: warp shuffle, one atomic per warp
  smax = warp_max(smax);
  if ((threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0)
    atomic_max_nonneg(&a.status->max_speed_bits, smax);
  if (__any_sync(0xffffffffu, bad) &&
      (threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0)
    atomicOr(&a.status->error_word, AXB_EW_NAN_FLUX);
}

} // namespace axb
