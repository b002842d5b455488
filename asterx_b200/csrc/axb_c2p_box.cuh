// Device side of the box recovery (AsterX_Con2PrimGroup,
// AsterX/schedule.ccl:119-165): the argument block, curl A -> dB_stag, the
// per-cell con2prim driver with its Noble -> Palenzuela -> entropy ->
// atmosphere cascade (AsterX/src/con2prim.cxx:73-454) and the recovery
// kernels, shared by the single-box launches (axb_poststep.cu), the batched
// ones (axb_c2p_batch.cu) and the independent-cell recovery
// (axb_c2p_cells.cu); each translation unit instantiates the kernels it
// launches.  Every file that includes this is compiled without multiply-add
// contraction (asterx_b200/build.py), so all kernels give a cell the same
// bits.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>

#include "axb_batch.cuh"
#include "axb_c2p.cuh"
#include "axb_internal.hxx"

namespace axb {

struct C2PBoxArgs {
  BoxDev b;
  // inputs / outputs (all cell-centred unless noted)
  const double *Avec[3];   // edges
  double *dBstag[3];       // faces
  const double *alp, *g[6];
  double *dens, *mom[3], *tau, *DYe, *DEnt, *dB[3];
  double *rho, *vel[3], *eps, *press, *temperature, *Ye, *entropy, *Bvec[3];
  double *saved_rho, *saved_vel[3], *saved_eps, *saved_Ye;
  double *zvec[3], *svec[3], *flag;
  // settings
  C2PParams cp;
  int c2p_prime, c2p_second, excise, thermal_eos_atmo, use_press_atmo;
  int use_entropy_fix; // the entropy scheme after both schemes failed
  int atmo_uniform;
  Atmo atmo_const; // when atmo_uniform
  double rho_abs_min, r_atmo, n_rho_atmo, p_atmo, n_press_atmo, t_atmo,
      n_temp_atmo, Ye_atmo, atmo_tol;
  double gamma_noble, Zmin;
  EosPoly poly;
  int want_hist;
  // ghost layers across each face set that curl A covers: 1 (the next RHS
  // reads one), 3 with upwind CT (its edge reconstructions reach three)
  int bext;
  // learned guess (x = h W, W) of each interior cell, (i, j, k) at
  // ((k - ng) n_y + j - ng) n_x + i - ng, and the half-width of the
  // Palenzuela bracket around x; read only by the GUESS kernels
  const float2 *guess;
  double bracket;
  DevStatus *status;
};

template <class EOS>
AXB_D void run_solver_guess(int which, const EOS &eos, const C2PBoxArgs &a, const Atmo &atmo,
                            Prim &pv, Prim &seeds, Cons &cv, const sym3 &glo, Report &rep,
                            double zguess, double vsqguess, double xlo, double xhi) {
  if (which == AXB_C2P_NOBLE)
    noble_solve(eos, a.cp, atmo, a.gamma_noble, a.Zmin, pv, seeds, cv, glo, rep, zguess,
                vsqguess);
  else if (which == AXB_C2P_PALENZUELA)
    palenzuela_solve(eos, a.cp, atmo, pv, cv, glo, rep, xlo, xhi);
  else if (which == AXB_C2P_ENTROPY)
    entropy_solve(eos, a.cp, atmo, pv, cv, glo, rep);
}

// ComputeStaggeredB<dir> (AsterX/src/computeBfromA.cxx:20-56) on the faces
// [ng, ng+n] along d and [ng-e, ng+n+e-1] across, e = bext ghost layers
// (which the next RHS needs and the reference obtains by SYNC).
AXB_D void bstag_body(const C2PBoxArgs &a, const uint3 bid) {
  const BoxDev &b = a.b;
  const int ng = b.ng;
  const int e = a.bext;
  int i, j;
  const int k = ng - e + bid.z;
  if (!b.row_ij(ng - e, b.n[0] + 2 * e, ng - e, b.n[1] + 2 * e, bid, i, j))
    return;
  const long long I = b.at(i, j, k);
  const long long ipjk = I + 1, ijpk = I + b.sy, ijkp = I + b.sz;
  const double *Ax = a.Avec[0], *Ay = a.Avec[1], *Az = a.Avec[2];
  const bool in_i = i >= ng && i <= ng + b.n[0];
  const bool in_j = j >= ng && j <= ng + b.n[1];
  const bool in_k = k >= ng && k <= ng + b.n[2];
  // x-faces: vertex in x, cells in y, z
  if (in_i && j <= ng + b.n[1] + e - 1 && k <= ng + b.n[2] + e - 1)
    a.dBstag[0][I] = b.idx[1] * (Az[ijpk] - Az[I]) - b.idx[2] * (Ay[ijkp] - Ay[I]);
  if (in_j && i <= ng + b.n[0] + e - 1 && k <= ng + b.n[2] + e - 1)
    a.dBstag[1][I] = b.idx[2] * (Ax[ijkp] - Ax[I]) - b.idx[0] * (Az[ipjk] - Az[I]);
  if (in_k && i <= ng + b.n[0] + e - 1 && j <= ng + b.n[1] + e - 1)
    a.dBstag[2][I] = b.idx[0] * (Ay[ipjk] - Ay[I]) - b.idx[1] * (Ax[ijpk] - Ax[I]);
}

template <class EOS>
AXB_D Atmo cell_atmosphere(const C2PBoxArgs &a, const EOS &eos, double x,
                           double y, double z) {
  // graded atmosphere (con2prim.cxx:81-133)
  const double r = sqrt(x * x + y * y + z * z);
  double rho_atm = (r > a.r_atmo) ? (a.rho_abs_min * pow((a.r_atmo / r), a.n_rho_atmo))
                                  : a.rho_abs_min;
  rho_atm = fmax(eos.rgrho.min, rho_atm);
  double press_atm, eps_atm, temp_atm = 0.0;
  if (a.thermal_eos_atmo) {
    if (a.use_press_atmo) {
      press_atm = (r > a.r_atmo) ? (a.p_atmo * pow(a.r_atmo / r, a.n_press_atmo)) : a.p_atmo;
      press_atm = fmax(eos.press_from_valid_rho_temp_ye(rho_atm, eos.rgtemp.min, a.Ye_atmo),
                       press_atm);
      eps_atm = eos.eps_from_valid_rho_press_ye(rho_atm, press_atm, a.Ye_atmo);
      temp_atm = eos.temp_from_valid_rho_eps_ye(rho_atm, eps_atm, a.Ye_atmo);
    } else {
      temp_atm = (r > a.r_atmo) ? (a.t_atmo * pow(a.r_atmo / r, a.n_temp_atmo)) : a.t_atmo;
      temp_atm = fmax(eos.rgtemp.min, temp_atm);
      press_atm = eos.press_from_valid_rho_temp_ye(rho_atm, temp_atm, a.Ye_atmo);
      eps_atm = eos.eps_from_valid_rho_temp_ye(rho_atm, temp_atm, a.Ye_atmo);
    }
  } else {
    const double gm1 = a.poly.gm1_from_valid_rho(rho_atm);
    eps_atm = a.poly.sed_from_valid_gm1(gm1);
    eps_atm = fmin(fmax(eos.rgeps.min, eps_atm), eos.rgeps.max);
    press_atm = eos.press_from_valid_rho_eps_ye(rho_atm, eps_atm, a.Ye_atmo);
  }
  const double entropy_atm = eos.kappa_from_valid_rho_eps_ye(rho_atm, eps_atm, a.Ye_atmo);
  return Atmo{rho_atm, eps_atm, a.Ye_atmo, press_atm, temp_atm, entropy_atm,
              rho_atm * (1 + a.atmo_tol)};
}

template <class EOS>
AXB_D void run_solver(int which, const EOS &eos, const C2PBoxArgs &a,
                      const Atmo &atmo, Prim &pv, Prim &seeds, Cons &cv,
                      const sym3 &glo, Report &rep) {
  if (which == AXB_C2P_NOBLE)
    noble_solve(eos, a.cp, atmo, a.gamma_noble, a.Zmin, pv, seeds, cv, glo, rep);
  else if (which == AXB_C2P_PALENZUELA)
    palenzuela_solve(eos, a.cp, atmo, pv, cv, glo, rep);
  else if (which == AXB_C2P_ENTROPY)
    entropy_solve(eos, a.cp, atmo, pv, cv, glo, rep);
}

// Both schemes failed (con2prim.cxx:308-416): the entropy scheme when
// use_entropy_fix, then, if that fails too (or without it), the failure
// treatment -- BH-interior values inside the mask, else atmosphere with the
// cell's B.  Returns the flag code; `failed` marks a cell nothing recovered.
template <class EOS>
AXB_D int after_both_failed(const EOS &eos, const C2PBoxArgs &a, const Atmo &atmo,
                            double mask_local, double sqrt_detg, const double (&Bup)[3],
                            Prim &pv, Prim &seeds, Cons &cv, const sym3 &glo,
                            bool &flag_local, bool &failed) {
  if (a.use_entropy_fix) {
    Report re;
    entropy_solve(eos, a.cp, atmo, pv, cv, glo, re);
    if (!re.failed())
      return AXB_C2P_ENTROPY_OK;
  }
  flag_local = false;
  failed = true;
  if (mask_local != 1.0) {
    bh_interior<false>(eos, a.cp, atmo, seeds, cv, glo);
    pv = seeds;
  } else {
    for (int q = 0; q < 3; ++q) {
      cv.dBvec[q] = sqrt_detg * Bup[q];
      pv.Bvec[q] = Bup[q];
    }
    atmo.set(pv, cv, glo);
  }
  return AXB_C2P_FAIL;
}

// One cell of AsterX_Con2Prim_typeEoS (con2prim.cxx:81-453), preceded by
// AsterX_ComputedBFromdBstag (computeBfromA.cxx:67-85) for the same cell.
#ifndef AXB_C2P_MINB
#define AXB_C2P_MINB 4 // resident CTAs per SM the register budget must allow
#endif
#ifndef AXB_C2P_FAST_MINB
#define AXB_C2P_FAST_MINB 7 // the fast pass: fewer live values, more warps
#endif
//
// MODE C2P_FULL runs the whole cascade.  MODE C2P_FAST (Palenzuela as the
// first solver) runs the common path only and returns true, having written
// nothing, for a cell that needs anything else -- the excision / BH-interior
// treatment, a Palenzuela failure (and so the second solver), or a bracket
// that did not converge (and so the conservative-variable check); such a
// cell is then recovered by the full cascade in a second launch, from the
// same unmodified inputs, so every cell gets exactly the full cascade's
// result.  The rare paths' code stays out of the fast kernel and no warp of
// it waits on them.
//
// GUESS (with a.guess): the first solver starts from the learned guess --
// the Noble seeds Z = D x, v^2 = 1 - 1/W^2, or the Palenzuela bracket
// x (1 -+ bracket).  A guessed first attempt that fails returns C2P_RETRY
// having written nothing; the caller then runs the cell again without the
// guess (the plain seeds, as c2p_2DNoble.hxx:374-393 and
// c2p_1DPalenzuela.hxx:395-401 set them, and the plain cascade).
enum { C2P_FULL = 0, C2P_FAST = 1 };
enum { C2P_DONE = 0, C2P_DEFERRED = 1, C2P_RETRY = 2 };
template <class EOS, int MODE, bool GUESS = false>
AXB_D int c2p_cell(const C2PBoxArgs &a, const EOS &eos, const int i, const int j,
                   const int k, int &iters_first, bool &failed, bool use_guess = false) {
  constexpr bool FASTLIKE = MODE == C2P_FAST;
  const BoxDev &b = a.b;
  {
    const long long I = b.at(i, j, k);
    double dB[3];
    dB[0] = 0.5 * (a.dBstag[0][I] + a.dBstag[0][I + 1]);
    dB[1] = 0.5 * (a.dBstag[1][I] + a.dBstag[1][I + b.sy]);
    dB[2] = 0.5 * (a.dBstag[2][I] + a.dBstag[2][I + b.sz]);
    Atmo atmo;
    if (a.atmo_uniform) {
      atmo = a.atmo_const;
    } else {
      const double x = b.xmin[0] + (i - b.ng + 0.5) * b.dx[0];
      const double y = b.xmin[1] + (j - b.ng + 0.5) * b.dx[1];
      const double z = b.xmin[2] + (k - b.ng + 0.5) * b.dx[2];
      atmo = cell_atmosphere(a, eos, x, y, z);
    }
    // vertex-to-cell metric (aster_interp.hxx:23-36)
    auto v2c = [&](const double *f) {
      double s = 0.0;
      s += f[I];
      s += f[I + 1];
      s += f[I + b.sy];
      s += f[I + 1 + b.sy];
      s += f[I + b.sz];
      s += f[I + 1 + b.sz];
      s += f[I + b.sy + b.sz];
      s += f[I + 1 + b.sy + b.sz];
      return s / 8.0;
    };
    const double alp_avg = v2c(a.alp);
    const sym3 glo{v2c(a.g[0]), v2c(a.g[1]), v2c(a.g[2]),
                   v2c(a.g[3]), v2c(a.g[4]), v2c(a.g[5])};
    double mask_local = 1.0;
    const double spatial_detg = det3(glo);
    const double sqrt_detg = sqrt(spatial_detg);
    double v_up[3] = {a.saved_vel[0][I], a.saved_vel[1][I], a.saved_vel[2][I]};
    double v_low[3];
    lower3(glo, v_up, v_low);
    double zsq;
    const double vsq = dot3(v_low, v_up);
    if (vsq >= 1.0) {
      const double wlim = sqrt(1.0 + a.cp.vw_lim * a.cp.vw_lim);
      const double vlim = a.cp.vw_lim / wlim;
      for (int q = 0; q < 3; ++q) {
        v_up[q] *= vlim / sqrt(vsq);
        v_low[q] *= vlim / sqrt(vsq);
      }
      zsq = a.cp.vw_lim * a.cp.vw_lim;
    } else {
      zsq = vsq / (1.0 - vsq);
    }
    double wlor = sqrt(1.0 + zsq);
    Cons cv;
    cv.dens = a.dens[I];
    for (int q = 0; q < 3; ++q)
      cv.mom[q] = a.mom[q][I];
    cv.tau = a.tau[I];
    cv.DYe = a.DYe[I];
    cv.DEnt = a.DEnt[I];
    for (int q = 0; q < 3; ++q)
      cv.dBvec[q] = dB[q];
    const double isg = 1.0 / sqrt_detg;
    const double Bup[3] = {cv.dBvec[0] * isg, cv.dBvec[1] * isg, cv.dBvec[2] * isg};
    Prim pv;
    pv.set_nan();
    Prim seeds;
    seeds.rho = a.saved_rho[I];
    seeds.eps = a.saved_eps[I];
    seeds.Ye = a.saved_Ye[I];
    {
      double e = seeds.eps; // the reference clamps a copy, not the seed
      seeds.press = eos.press_from_valid_rho_eps_ye(seeds.rho, e, seeds.Ye);
    }
    seeds.temperature = a.temperature[I];
    seeds.entropy = 0.0; // only read by the excision path, filled there
    for (int q = 0; q < 3; ++q) {
      seeds.vel[q] = v_up[q];
      seeds.Bvec[q] = Bup[q];
      seeds.E[q] = 0.0;
    }
    seeds.w_lor = wlor;
    bool flag_local = true;
    int code = AXB_C2P_INIT;
    bool call_c2p = true;
    if (cv.dens <= sqrt_detg * atmo.rho_cut) {
      for (int q = 0; q < 3; ++q)
        pv.Bvec[q] = Bup[q];
      atmo.set(pv, cv, glo);
      atmo.set(seeds);
      code = AXB_C2P_ATMO;
      call_c2p = false;
    }
    if (alp_avg < a.cp.alp_thresh)
      mask_local = 0.0;
    if constexpr (FASTLIKE) {
      if (mask_local != 1.0)
        return C2P_DEFERRED;
    }
    if (MODE == C2P_FULL && a.excise && mask_local != 1.0) {
      seeds.entropy = eos.kappa_from_valid_rho_eps_ye(seeds.rho, seeds.eps, seeds.Ye);
      bh_interior<false>(eos, a.cp, atmo, seeds, cv, glo);
      pv = seeds;
      call_c2p = false;
    }
    double zguess = -1.0, vsqguess = -1.0, xlo = -1.0, xhi = -1.0;
    if constexpr (GUESS) {
      if (use_guess && call_c2p) {
        const long long ci =
            ((long long)(k - b.ng) * b.n[1] + (j - b.ng)) * b.n[0] + (i - b.ng);
        const float2 gs = a.guess[ci];
        const double x = gs.x, W = gs.y;
        zguess = cv.dens / sqrt_detg * x; // Z = rho h W^2 = D (h W)
        vsqguess = 1.0 - 1.0 / (W * W);
        xlo = x * (1.0 - a.bracket);
        xhi = x * (1.0 + a.bracket);
        if (!(zguess > 0.0 && zguess < 1e300 && vsqguess >= 0.0 && vsqguess < 1.0))
          zguess = vsqguess = xlo = xhi = -1.0;
      }
    }
    cons_floors(cv, glo);
    if constexpr (FASTLIKE) {
      if (call_c2p) {
        Report r1;
        code = AXB_C2P_PRIME;
        palenzuela_solve<EOS, true>(eos, a.cp, atmo, pv, cv, glo, r1, xlo, xhi);
        if (r1.failed())
          return C2P_DEFERRED; // REP_DEFER: every failure goes to the full cascade
        iters_first = r1.iters;
      }
    } else if (call_c2p) {
      Report r1, r2;
      code = AXB_C2P_PRIME;
      if (GUESS && zguess >= 0.0) {
        run_solver_guess(a.c2p_prime, eos, a, atmo, pv, seeds, cv, glo, r1, zguess, vsqguess,
                         xlo, xhi);
        if (r1.failed()) {
          iters_first = r1.iters;
          return C2P_RETRY;
        }
      } else {
        run_solver(a.c2p_prime, eos, a, atmo, pv, seeds, cv, glo, r1);
      }
      iters_first = r1.iters;
      if (r1.failed()) {
        code = AXB_C2P_SECOND;
        run_solver(a.c2p_second, eos, a, atmo, pv, seeds, cv, glo, r2);
      }
      if (r1.failed() && r2.failed())
        code = after_both_failed(eos, a, atmo, mask_local, sqrt_detg, Bup, pv, seeds, cv, glo,
                                 flag_local, failed);
      if ((mask_local != 1.0) && flag_local)
        bh_interior<true>(eos, a.cp, atmo, pv, cv, glo);
    }
    a.flag[I] = code;
    a.rho[I] = pv.rho;
    a.eps[I] = pv.eps;
    a.Ye[I] = pv.Ye;
    a.press[I] = pv.press;
    a.temperature[I] = pv.temperature;
    a.entropy[I] = pv.entropy;
    for (int q = 0; q < 3; ++q) {
      a.vel[q][I] = pv.vel[q];
      a.Bvec[q][I] = pv.Bvec[q];
    }
    wlor = pv.w_lor;
    const double hW2 = (pv.rho + pv.rho * pv.eps + pv.press) * wlor * wlor;
    for (int q = 0; q < 3; ++q) {
      if (a.zvec[q])
        a.zvec[q][I] = wlor * pv.vel[q];
      if (a.svec[q])
        a.svec[q][I] = hW2 * pv.vel[q];
    }
    a.dens[I] = cv.dens;
    for (int q = 0; q < 3; ++q)
      a.mom[q][I] = cv.mom[q];
    a.tau[I] = cv.tau;
    a.DYe[I] = cv.DYe;
    a.DEnt[I] = cv.DEnt;
    for (int q = 0; q < 3; ++q)
      if (a.dB[q])
        a.dB[q][I] = cv.dBvec[q];
    a.saved_rho[I] = pv.rho;
    for (int q = 0; q < 3; ++q)
      a.saved_vel[q][I] = pv.vel[q];
    a.saved_eps[I] = pv.eps;
    a.saved_Ye[I] = pv.Ye;
  }
  return C2P_DONE;
}

// Warp and block epilogue of a recovery launch: failure count, and the
// first solver's iteration histogram through shared memory (every thread of
// the block must arrive).
AXB_D void c2p_hist_init(const C2PBoxArgs &a, unsigned int *s_hist) {
  if (a.want_hist) {
    for (int q = threadIdx.x; q < 64; q += blockDim.x)
      s_hist[q] = 0;
    __syncthreads();
  }
}
AXB_D void c2p_epilogue(const C2PBoxArgs &a, unsigned int *s_hist, int iters_first,
                        bool failed) {
  const unsigned nfail = __popc(__ballot_sync(0xffffffffu, failed));
  if (nfail && (threadIdx.x % 32) == 0) {
    atomicAdd(&a.status->c2p_fail_count, nfail);
    atomicOr(&a.status->error_word, AXB_EW_C2P_FAIL);
  }
  if (a.want_hist) {
    if (iters_first >= 0)
      atomicAdd(&s_hist[min(iters_first, 63)], 1u);
    __syncthreads();
    for (int q = threadIdx.x; q < 64; q += blockDim.x)
      if (s_hist[q])
        atomicAdd(&a.status->c2p_iter_hist[q], (unsigned long long)s_hist[q]);
  }
}

// The full cascade on one cell; with GUESS a failed guessed attempt is
// followed by the plain one, and the cell's first-solver iterations count
// both attempts.
template <class EOS, bool GUESS>
AXB_D void c2p_cell_full(const C2PBoxArgs &a, const EOS &eos, int i, int j, int k,
                         int &iters_first, bool &failed) {
  if constexpr (GUESS) {
    int it0 = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      const int rc =
          c2p_cell<EOS, C2P_FULL, true>(a, eos, i, j, k, iters_first, failed, attempt == 0);
      if (rc != C2P_RETRY) {
        if (attempt == 1 && iters_first >= 0)
          iters_first += it0;
        return;
      }
      it0 = iters_first;
    }
  } else {
    c2p_cell<EOS, C2P_FULL>(a, eos, i, j, k, iters_first, failed);
  }
}

template <class EOS, bool GUESS = false>
AXB_D void c2p_box_body(const C2PBoxArgs &a, const EOS &eos, const uint3 bid) {
  __shared__ unsigned int s_hist[64];
  c2p_hist_init(a, s_hist);
  int i, j;
  const int k = a.b.ng + bid.z;
  const bool in_range = a.b.row_ij(a.b.ng, a.b.n[0], a.b.ng, a.b.n[1], bid, i, j);
  int iters_first = -1;
  bool failed = false;
  if (in_range)
    c2p_cell_full<EOS, GUESS>(a, eos, i, j, k, iters_first, failed);
  c2p_epilogue(a, s_hist, iters_first, failed);
}
template <class EOS, bool GUESS = false>
__global__ void __launch_bounds__(128, AXB_C2P_MINB)
    k_c2p_box(const C2PBoxArgs a, const EOS eos) {
  c2p_box_body<EOS, GUESS>(a, eos, blockIdx);
}

// Deferred cells of a fast pass: the count, then one entry per cell,
// i | j << 15 | k << 30 | box << 45 (box 0 for a single box).
struct C2PQueue {
  unsigned long long *count;
  unsigned long long *cell;
};
constexpr int C2P_QUEUE_MAX_EXTENT = 1 << 15; // per axis, ghosts included
constexpr int C2P_QUEUE_MAX_BOXES = 1 << 19;

// Append the deferred cells of a warp to the queue (one atomic per warp;
// every lane of the warp must call).
AXB_D void queue_deferred(const C2PQueue &q, bool defer, int i, int j, int k, int box) {
  const unsigned m = __ballot_sync(0xffffffffu, defer);
  if (m) {
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader)
      base = atomicAdd(q.count, (unsigned long long)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (defer)
      q.cell[base + __popc(m & ((1u << lane) - 1u))] =
          (unsigned long long)i | ((unsigned long long)j << 15) |
          ((unsigned long long)k << 30) | ((unsigned long long)box << 45);
  }
}

// Fast pass over one tile: the common path, deferred cells appended to the
// queue (warp-aggregated).
template <class EOS, bool GUESS = false>
AXB_D void c2p_fast_body(const C2PBoxArgs &a, const EOS &eos, const uint3 bid, int box,
                         const C2PQueue &q) {
  __shared__ unsigned int s_hist[64];
  c2p_hist_init(a, s_hist);
  int i, j;
  const int k = a.b.ng + bid.z;
  const bool in_range = a.b.row_ij(a.b.ng, a.b.n[0], a.b.ng, a.b.n[1], bid, i, j);
  int iters_first = -1;
  bool failed = false;
  bool defer = false;
  if (in_range)
    defer = c2p_cell<EOS, C2P_FAST, GUESS>(a, eos, i, j, k, iters_first, failed, GUESS) ==
            C2P_DEFERRED;
  queue_deferred(q, defer, i, j, k, box);
  c2p_epilogue(a, s_hist, iters_first, failed);
}

// The full cascade over the queued cells; `args_of(box)` gives the box's
// argument block.  Every thread runs the same number of rounds, so the
// warp-level epilogue sees full warps.
template <class EOS, class ArgsOf, bool GUESS = false>
AXB_D void c2p_deferred_body(const ArgsOf &args_of, const EOS &eos, const C2PQueue &q) {
  __shared__ unsigned int s_hist[64];
  const C2PBoxArgs &a0 = args_of(0);
  const bool want_hist = a0.want_hist;
  DevStatus *const status = a0.status;
  if (want_hist) {
    for (int t = threadIdx.x; t < 64; t += blockDim.x)
      s_hist[t] = 0;
    __syncthreads();
  }
  const unsigned long long n = *q.count;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long rounds = (n + stride - 1) / stride;
  for (unsigned long long r = 0; r < rounds; ++r) {
    const unsigned long long e = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
    int iters_first = -1;
    bool failed = false;
    if (e < n) {
      const unsigned long long v = q.cell[e];
      const int i = int(v & 0x7fff), j = int((v >> 15) & 0x7fff), k = int((v >> 30) & 0x7fff);
      c2p_cell_full<EOS, GUESS>(args_of(int(v >> 45)), eos, i, j, k, iters_first, failed);
    }
    const unsigned nfail = __popc(__ballot_sync(0xffffffffu, failed));
    if (nfail && (threadIdx.x % 32) == 0) {
      atomicAdd(&status->c2p_fail_count, nfail);
      atomicOr(&status->error_word, AXB_EW_C2P_FAIL);
    }
    if (want_hist && iters_first >= 0)
      atomicAdd(&s_hist[min(iters_first, 63)], 1u);
  }
  if (want_hist) {
    __syncthreads();
    for (int t = threadIdx.x; t < 64; t += blockDim.x)
      if (s_hist[t])
        atomicAdd(&status->c2p_iter_hist[t], (unsigned long long)s_hist[t]);
  }
}

template <class EOS, bool GUESS = false>
__global__ void __launch_bounds__(128, AXB_C2P_FAST_MINB)
    k_c2p_fast(const C2PBoxArgs a, const EOS eos, const C2PQueue q) {
  c2p_fast_body<EOS, GUESS>(a, eos, blockIdx, 0, q);
}

template <class EOS, bool GUESS = false>
__global__ void __launch_bounds__(128, AXB_C2P_MINB)
    k_c2p_deferred(const C2PBoxArgs a, const EOS eos, const C2PQueue q) {
  auto args_of = [&](int) -> const C2PBoxArgs & { return a; };
  c2p_deferred_body<EOS, decltype(args_of), GUESS>(args_of, eos, q);
}

// whether a box's extent fits the queue's packing
inline bool c2p_queue_fits(const axb_box &b) {
  for (int d = 0; d < 3; ++d)
    if (b.n[d] + 2 * b.ng + 1 > C2P_QUEUE_MAX_EXTENT)
      return false;
  return true;
}
} // namespace axb

namespace axb {
// The uniform atmosphere of a box inside r_atmo, on the host (the device
// form is cell_atmosphere).
template <class EOS>
Atmo host_atmosphere(const C2PBoxArgs &a, const EOS &eos) {
  double rho_atm = std::fmax(eos.rgrho.min, a.rho_abs_min);
  double press_atm, eps_atm, temp_atm = 0.0;
  if (a.thermal_eos_atmo) {
    if (a.use_press_atmo) {
      press_atm = std::fmax(eos.press_from_valid_rho_temp_ye(rho_atm, eos.rgtemp.min, a.Ye_atmo),
                            a.p_atmo);
      eps_atm = eos.eps_from_valid_rho_press_ye(rho_atm, press_atm, a.Ye_atmo);
      temp_atm = eos.temp_from_valid_rho_eps_ye(rho_atm, eps_atm, a.Ye_atmo);
    } else {
      temp_atm = std::fmax(eos.rgtemp.min, a.t_atmo);
      press_atm = eos.press_from_valid_rho_temp_ye(rho_atm, temp_atm, a.Ye_atmo);
      eps_atm = eos.eps_from_valid_rho_temp_ye(rho_atm, temp_atm, a.Ye_atmo);
    }
  } else {
    const double gm1 = a.poly.gm1_from_valid_rho(rho_atm);
    eps_atm = a.poly.sed_from_valid_gm1(gm1);
    eps_atm = std::fmin(std::fmax(eos.rgeps.min, eps_atm), eos.rgeps.max);
    press_atm = eos.press_from_valid_rho_eps_ye(rho_atm, eps_atm, a.Ye_atmo);
  }
  const double entropy_atm = eos.kappa_from_valid_rho_eps_ye(rho_atm, eps_atm, a.Ye_atmo);
  return Atmo{rho_atm, eps_atm, a.Ye_atmo, press_atm, temp_atm, entropy_atm,
              rho_atm * (1 + a.atmo_tol)};
}

// host helpers (axb_poststep.cu)
int check_box_c2p(const axb_box *b);
C2PParams make_c2p_params(const axb_params &p);
int fill_c2p_args(axb_ctx *c, const axb_box *box, const axb_fields *f,
                  const axb_params *p, const axb_eos *eos, C2PBoxArgs &a);
} // namespace axb
