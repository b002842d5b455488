// RHS kernels (see axb_rhs.cuh for the overview).
#pragma once

#include "axb_rhs.cuh"

#ifndef AXB_FLUX_STASH
#define AXB_FLUX_STASH 1 // the left face state in shared memory (face_fluxes)
#endif

namespace axb {

template <int N>
AXB_D void load_pencil(const double *__restrict__ f, long long I, long long s,
                       double (&q)[N]) {
#pragma unroll
  for (int m = 0; m < N; ++m)
    q[m] = __ldg(f + I + (m - N / 2) * s);
}

AXB_D void prefetch_l2(const double *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

AXB_D double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---------------------------------------------------------------------------
// Shared pieces of the flux passes.
// ---------------------------------------------------------------------------

// Reconstruct the NREC variables of the cell at I (stride sd along DIR).
template <int DIR, int RECON>
AXB_D void recon_cell_all(const RhsArgs &a, const double *const (&fld)[NREC],
                          long long I, long long sd, double (&lo)[NREC],
                          double (&up)[NREC]) {
  double pr[5], vd[5];
  load_pencil<5>(a.press, I, sd, pr);
  load_pencil<5>(a.vel[DIR], I, sd, vd);
#pragma unroll
  for (int v = 0; v < NREC; ++v) {
    double q[5];
    if (v == R_PRESS && !a.rec_temp) {
#pragma unroll
      for (int m = 0; m < 5; ++m) q[m] = pr[m];
    } else if (v == R_VX + DIR && a.recvar == AXB_RECVAR_V) {
#pragma unroll
      for (int m = 0; m < 5; ++m) q[m] = vd[m];
    } else {
      load_pencil<5>(fld[v], I, sd, q);
    }
    const CellLoUp r = recon_cell<RECON>(q, pr, vd, v == R_RHO, a.rp);
    lo[v] = r.lo;
    up[v] = r.up;
  }
}

// The face between the cells at I - sd and I, given the left state L (upper
// values of the left cell) and the right state R (lower values of the right
// cell): low-order redo of a side with a non-positive rho, entropy, Ye or
// thermodynamic variable (fluxes.cxx:263-343), face metric, both states'
// conserved variables, fluxes and fast speeds, and the Riemann flux
// (HLLE or LxF, fluxes.cxx:162-200).  Stores the two transverse B fluxes
// when asked.
template <int DIR, bool UCT, class EOS>
AXB_D void face_fluxes(const RhsArgs &a, const EOS &eos,
                       const double *const (&fld)[NREC], long long I, long long sd,
                       double (&L)[NREC], double (&R)[NREC], double (&F)[10],
                       double &smax, bool &bad) {
  constexpr int D1 = (DIR + 1) % 3, D2 = (DIR + 2) % 3;
  const bool lo0 = (L[R_RHO] <= 0.0) || (L[R_ENT] <= 0.0) ||
                   (L[R_YE] <= 0.0) || (L[R_PRESS] <= 0.0);
  const bool lo1 = (R[R_RHO] <= 0.0) || (R[R_ENT] <= 0.0) ||
                   (R[R_YE] <= 0.0) || (R[R_PRESS] <= 0.0);
  if (lo0 || lo1) {
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
  const double Bdir = __ldg(a.dBstag[DIR] + I) * m.isqrtg;
  SideOut sL, sR;
  side_physics<DIR, UCT>(m, L, Bdir, eos, a.rec_temp, a.recvar, sL);
  // (y and z passes) the left state's conserved variables and fluxes wait in
  // shared memory while the right state is formed: held in registers, the
  // two states together push the pencil march past its register budget
  // (measured at 256^3: y 3.40 -> 3.21 ms, z 4.06 -> 3.79 ms; the x pass,
  // which carries less, was not faster with it)
  constexpr bool stash = AXB_FLUX_STASH && DIR != 0;
  volatile double *sl = nullptr;
  if constexpr (stash) {
    __shared__ double s_left[20][128];
    sl = &s_left[0][threadIdx.y * blockDim.x + threadIdx.x];
#pragma unroll
    for (int v = 0; v < 10; ++v) {
      sl[128 * v] = sL.U[v];
      sl[128 * (10 + v)] = sL.F[v];
    }
  }
  auto uL = [&](int v) -> double {
    if constexpr (stash)
      return sl[128 * v];
    else
      return sL.U[v];
  };
  auto fL = [&](int v) -> double {
    if constexpr (stash)
      return sl[128 * (10 + v)];
    else
      return sL.F[v];
  };
  side_physics<DIR, UCT>(m, R, Bdir, eos, a.rec_temp, a.recvar, sR);
  const double cmax = fmax(0.0, fmax(fmax(sL.lam_p, sL.lam_m), fmax(sR.lam_p, sR.lam_m)));
  const double cmin = fmin(0.0, fmin(fmin(sL.lam_p, sL.lam_m), fmin(sR.lam_p, sR.lam_m)));
  smax = fmax(smax, fmax(cmax, -cmin));
  if (a.flux_type == AXB_FLUX_HLLE) {
    const double icpm = 1 / (cmax - cmin);
#pragma unroll
    for (int v = 0; v < 10; ++v)
      F[v] = hlle_flux(cmax, cmin, icpm, uL(v), sR.U[v], fL(v), sR.F[v]);
  } else {
    const double ch = fmax(cmax, -cmin);
#pragma unroll
    for (int v = 0; v < 10; ++v)
      F[v] = laxf_flux(ch, uL(v), sR.U[v], fL(v), sR.F[v]);
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
  if constexpr (UCT) {
    // upwind-CT face data (fluxes.cxx:776-794): the bounding speeds and the
    // transverse vtilde averaged with them
    const double amax = cmax, amin = -cmin;
    a.uct[4 * DIR + 0][I] = (amax * sL.vt1 + amin * sR.vt1) / (amax + amin);
    a.uct[4 * DIR + 1][I] = (amax * sL.vt2 + amin * sR.vt2) / (amax + amin);
    a.uct[4 * DIR + 2][I] = amax;
    a.uct[4 * DIR + 3][I] = amin;
  }
}

// Fold F(face c+1) - F(face c) into the partial divergence of cell c (at I),
// in the reference's summation order (rhs.cxx:188-207): x writes, y adds,
// z adds and forms the RHS.  Returns true when the z pass formed a
// non-finite hydro RHS (the reference asserts there, rhs.cxx:199-206).
template <int DIR>
AXB_D bool fold_divergence(const RhsArgs &a, long long I, double idxd,
                           const double (&Fhi)[NHYDRO], const double (&Flo)[NHYDRO]) {
  bool bad = false;
#pragma unroll
  for (int v = 0; v < NHYDRO; ++v) {
    const double dF = Fhi[v] - Flo[v];
    if (DIR == 0) {
      a.acc[v][I] = idxd * dF;
    } else if (DIR == 1) {
      a.acc[v][I] = a.acc[v][I] + idxd * dF;
    } else {
      const double r = a.rhs[v][I] + (-(a.acc[v][I] + idxd * dF));
      if (a.fuse_stage)
        a.st_uk[v][I] = stage_combine(a.st_alpha, a.st_un[v][I], a.st_beta,
                                      a.st_uk[v][I], a.st_gdt, r);
      else
        a.rhs[v][I] = r;
      bad |= !isfinite(r);
    }
  }
  return bad;
}

AXB_D void flux_status(const RhsArgs &a, double smax, bool bad, bool bad_rhs = false) {
  // characteristic-speed maximum: warp shuffle, one atomic per warp
  smax = warp_max(smax);
  const bool lead = (threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0;
  if (lead)
    atomic_max_nonneg(&a.status->max_speed_bits, smax);
  const bool any_bad = __any_sync(0xffffffffu, bad);
  const bool any_rhs = __any_sync(0xffffffffu, bad_rhs);
  if (lead && (any_bad || any_rhs))
    atomicOr(&a.status->error_word,
             (any_bad ? AXB_EW_NAN_FLUX : 0u) | (any_rhs ? AXB_EW_NAN_RHS : 0u));
}

#ifndef AXB_FLUX_MINB
#define AXB_FLUX_MINB 4 // resident CTAs per SM the register budget must allow
#endif
#ifndef AXB_FLUX_X_MINB
#define AXB_FLUX_X_MINB 4
#endif
#ifndef AXB_FLUX_SMEM_CARRY
#define AXB_FLUX_SMEM_CARRY 1
#endif
#ifndef AXB_FLUX_PREFETCH
#define AXB_FLUX_PREFETCH 1 // steps of L2 prefetch ahead of the march (0: none)
#endif
#ifndef AXB_FLUX_PF_RECON
#define AXB_FLUX_PF_RECON 1
#endif
#ifndef AXB_FLUX_PF_ACC
#define AXB_FLUX_PF_ACC 1
#endif

// ---------------------------------------------------------------------------
// k_flux_pass (y and z): one thread marches one pencil segment along DIR.
// Per step it reconstructs one cell (both interface values, ReconX per-cell
// formulas), forms the face between the previous cell and this one, and
// folds F(face) - F(face-1) into the partial divergence of the previous cell.
// Threads of a warp are adjacent along x, so every load is a coalesced
// 256-byte row.
// Transverse range: cells [ng-1, ng+n] (one ghost layer each side, needed
// by the edge electric field); faces along DIR: [ng, ng+n].
// ---------------------------------------------------------------------------
template <int DIR, int RECON, class EOS, bool UCT = false>
AXB_D void flux_pass_body(const RhsArgs &a, const EOS &eos, const int &seglen, const uint3 bid) {
  static_assert(DIR != 0, "the x pass is k_flux_x");
  constexpr int D1 = (DIR + 1) % 3, D2 = (DIR + 2) % 3;
  constexpr int T0 = 0;
  constexpr int T1 = (DIR == 2) ? 1 : 2;
  const BoxDev &b = a.b;
  const int ng = b.ng;
  constexpr int te = UCT ? 3 : 1; // transverse ghost layers covered
  int t0, t1;
  bool active;
  if (b.packed) {
    // (batched small boxes) the block's threads walk the transverse plane
    // [ng-te, ng+n+te-1]^2 row after row, so short rows leave no lane idle
    const int w0 = b.n[T0] + 2 * te;
    const int flat = bid.x * (blockDim.x * blockDim.y) + threadIdx.y * blockDim.x + threadIdx.x;
    t0 = ng - te + flat % w0;
    t1 = ng - te + flat / w0;
    active = flat < w0 * (b.n[T1] + 2 * te);
  } else {
    t0 = ng - te + bid.x * blockDim.x + threadIdx.x;
    t1 = ng - te + bid.y * blockDim.y + threadIdx.y;
    active = (t0 <= ng + b.n[T0] + te - 1) && (t1 <= ng + b.n[T1] + te - 1);
  }
  double smax = 0.0;
  bool bad = false, bad_rhs = false;
  if (active) {
    const bool trans_int = (t0 >= ng) && (t0 < ng + b.n[T0]) && (t1 >= ng) &&
                           (t1 < ng + b.n[T1]);
    const int f0 = ng + bid.z * seglen;
    const int flast = min(f0 + seglen, ng + b.n[DIR]);
    const long long sd = b.stride(DIR);
    int ijk[3];
    ijk[T0] = t0;
    ijk[T1] = t1;
    ijk[DIR] = f0 - 1;
    long long I = b.at(ijk[0], ijk[1], ijk[2]);
    const double *const fld[NREC] = {a.rho,     a.entropy, a.Ye,       a.thermo,
                                     a.recv[0], a.recv[1], a.recv[2], a.Bvec[D1],
                                     a.Bvec[D2]};
    const double idxd = b.idx[DIR];
#if AXB_FLUX_SMEM_CARRY
    // the state carried from one cell to the next (upper interface values
    // of the previous cell, flux of the previous face) lives in shared
    // memory: in registers it pushed the march beyond its register budget
    // and into local-memory spills
    __shared__ double s_carry[NREC + NHYDRO][128];
    const int tl = threadIdx.y * blockDim.x + threadIdx.x;
#define AXB_UPL(v) s_carry[v][tl]
#define AXB_FPREV(v) s_carry[NREC + (v)][tl]
#else
    double upL[NREC];
    double Fprev[NHYDRO];
#define AXB_UPL(v) upL[v]
#define AXB_FPREV(v) Fprev[v]
#endif
    for (int c = f0 - 1; c <= flast; ++c, I += sd) {
#if AXB_FLUX_PREFETCH > 0
      // L2 prefetch of the rows the march first touches AXB_FLUX_PREFETCH
      // steps ahead: the new stencil row of every reconstructed variable,
      // the face metric's two vertex rows, the face's staggered B and the
      // partial divergences (and RHS) it will accumulate into; all of them
      // within the rows this segment reads anyway
      if (c + AXB_FLUX_PREFETCH <= flast) {
        const long long J = I + AXB_FLUX_PREFETCH * sd;
#if AXB_FLUX_PF_RECON
#pragma unroll
        for (int v = 0; v < NREC; ++v)
          prefetch_l2(fld[v] + J + 2 * sd);
#endif
        constexpr int D1 = (DIR + 1) % 3, D2 = (DIR + 2) % 3;
        const long long so = (D1 == 0) ? b.stride(D2) : b.stride(D1);
        prefetch_l2(a.alp + J);
        prefetch_l2(a.alp + J + so);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          prefetch_l2(a.beta[q] + J);
          prefetch_l2(a.beta[q] + J + so);
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          prefetch_l2(a.g[q] + J);
          prefetch_l2(a.g[q] + J + so);
        }
        prefetch_l2(a.dBstag[DIR] + J);
        if (AXB_FLUX_PF_ACC && trans_int) {
#pragma unroll
          for (int v = 0; v < NHYDRO; ++v) {
            prefetch_l2(a.acc[v] + J - sd);
            if (DIR == 2)
              prefetch_l2(a.rhs[v] + J - sd);
          }
        }
      }
#endif
      double lo[NREC], up[NREC];
      recon_cell_all<DIR, RECON>(a, fld, I, sd, lo, up);
      if (c >= f0) {
        // face c: left state = upper values of cell c-1, right = lower of c
        double L[NREC], R[NREC], F[10];
#pragma unroll
        for (int v = 0; v < NREC; ++v) {
          L[v] = AXB_UPL(v);
          R[v] = lo[v];
        }
        face_fluxes<DIR, UCT>(a, eos, fld, I, sd, L, R, F, smax, bad);
        if (c > f0 && trans_int) {
          double Fc[NHYDRO], Fp[NHYDRO];
#pragma unroll
          for (int v = 0; v < NHYDRO; ++v) {
            Fc[v] = F[v];
            Fp[v] = AXB_FPREV(v);
          }
          bad_rhs |= fold_divergence<DIR>(a, I - sd, idxd, Fc, Fp);
        }
#pragma unroll
        for (int v = 0; v < NHYDRO; ++v)
          AXB_FPREV(v) = F[v];
      }
#pragma unroll
      for (int v = 0; v < NREC; ++v)
        AXB_UPL(v) = up[v];
    }
#undef AXB_UPL
#undef AXB_FPREV
  }
  flux_status(a, smax, bad, bad_rhs);
}
template <int DIR, int RECON, class EOS, bool UCT = false>
__global__ void __launch_bounds__(128, AXB_FLUX_MINB)
    k_flux_pass(const RhsArgs a, const EOS eos, const int seglen) {
  flux_pass_body<DIR, RECON, EOS, UCT>(a, eos, seglen, blockIdx);
}

// ---------------------------------------------------------------------------
// k_flux_x: the x pass with the lanes of a warp along x, so that every
// stencil load is a coalesced row segment (a thread marching along x would
// touch 32 rows per load and lose its sectors before coming back to them).
// Each warp owns one (y, z) row and walks it in chunks of 32 cells that
// overlap by two: lane l reconstructs cell c0 + l once, takes the left state
// of its face (c0 + l) from lane l - 1 by shuffle, computes the face, and
// takes the flux of face c0 + l + 1 from lane l + 1 to form the divergence
// of its cell.  Lanes 1..31 compute faces, lanes 1..30 divergences; a chunk
// advances 30 cells.
// ---------------------------------------------------------------------------
template <int RECON, class EOS, bool UCT = false>
AXB_D void flux_x_body(const RhsArgs &a, const EOS &eos, const uint3 bid) {
  const BoxDev &b = a.b;
  const int ng = b.ng;
  const int lane = threadIdx.x & 31;
  const int warp = (bid.x * blockDim.x + threadIdx.x) >> 5;
  constexpr int te = UCT ? 3 : 1; // transverse ghost layers covered
  const int ny = b.n[1] + 2 * te; // rows j, k in [ng-te, ng+n+te-1]
  const int nz = b.n[2] + 2 * te;
  double smax = 0.0;
  bool bad = false;
  if (warp < ny * nz) { // warp-uniform
    const int j = ng - te + warp % ny;
    const int k = ng - te + warp / ny;
    const bool trans_int = (j >= ng) && (j < ng + b.n[1]) && (k >= ng) && (k < ng + b.n[2]);
    const double *const fld[NREC] = {a.rho,     a.entropy, a.Ye,      a.thermo, a.recv[0],
                                     a.recv[1], a.recv[2], a.Bvec[1], a.Bvec[2]};
    const double idxd = b.idx[0];
    const long long row = b.at(0, j, k);
    const int clast = ng + b.n[0]; // last cell needed (right state of the last face)
    for (int c0 = ng - 1; c0 < ng + b.n[0] - 1; c0 += 30) {
      const int c = c0 + lane;
      const bool has_cell = c <= clast;
      const long long I = row + c;
      double lo[NREC], up[NREC];
      if (has_cell) {
        recon_cell_all<0, RECON>(a, fld, I, 1, lo, up);
      } else {
#pragma unroll
        for (int v = 0; v < NREC; ++v)
          lo[v] = up[v] = 0.0;
      }
      double L[NREC], R[NREC], F[10];
#pragma unroll
      for (int v = 0; v < NREC; ++v) {
        L[v] = __shfl_up_sync(0xffffffffu, up[v], 1);
        R[v] = lo[v];
      }
      const bool has_face = lane >= 1 && has_cell; // face c in [ng, ng+n]
      if (has_face) {
        face_fluxes<0, UCT>(a, eos, fld, I, 1, L, R, F, smax, bad);
      } else {
#pragma unroll
        for (int v = 0; v < 10; ++v)
          F[v] = 0.0;
      }
      double Fhi[NHYDRO], Flo[NHYDRO];
#pragma unroll
      for (int v = 0; v < NHYDRO; ++v) {
        Flo[v] = F[v];
        Fhi[v] = __shfl_down_sync(0xffffffffu, F[v], 1);
      }
      // cell c's divergence needs faces c and c+1
      if (trans_int && lane >= 1 && lane <= 30 && c < ng + b.n[0])
        fold_divergence<0>(a, I, idxd, Fhi, Flo);
    }
  }
  flux_status(a, smax, bad);
}
template <int RECON, class EOS, bool UCT = false>
__global__ void __launch_bounds__(128, AXB_FLUX_X_MINB)
    k_flux_x(const RhsArgs a, const EOS eos) {
  flux_x_body<RECON, EOS, UCT>(a, eos, blockIdx);
}

} // namespace axb
