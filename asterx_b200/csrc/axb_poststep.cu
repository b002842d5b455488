// PostStep group (AsterX_Con2PrimGroup, AsterX/schedule.ccl:119-165):
// curl A -> dB_stag, face-to-cell dB, and the con2prim driver with its
// Noble -> Palenzuela -> atmosphere cascade (AsterX/src/con2prim.cxx:73-454).
// Also the RK stage update and the periodic ghost fill of one box.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <limits>

#include "axb_batch.cuh"
#include "axb_c2p.cuh"
#include "axb_internal.hxx"
#include "axb_mlp.cuh"

using namespace axb;

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
  DevStatus *status;
};

// ComputeStaggeredB<dir> (AsterX/src/computeBfromA.cxx:20-56) on the faces
// [ng, ng+n] along d and [ng-1, ng+n] across (one ghost layer, which the next
// RHS needs and the reference obtains by SYNC).
AXB_D void bstag_body(const C2PBoxArgs &a, const uint3 bid) {
  const BoxDev &b = a.b;
  const int ng = b.ng;
  int i, j;
  const int k = ng - 1 + bid.z;
  if (!b.row_ij(ng - 1, b.n[0] + 2, ng - 1, b.n[1] + 2, bid, i, j))
    return;
  const long long I = b.at(i, j, k);
  const long long ipjk = I + 1, ijpk = I + b.sy, ijkp = I + b.sz;
  const double *Ax = a.Avec[0], *Ay = a.Avec[1], *Az = a.Avec[2];
  const bool in_i = i >= ng && i <= ng + b.n[0];
  const bool in_j = j >= ng && j <= ng + b.n[1];
  const bool in_k = k >= ng && k <= ng + b.n[2];
  // x-faces: vertex in x, cells in y, z
  if (in_i && j <= ng + b.n[1] && k <= ng + b.n[2])
    a.dBstag[0][I] = b.idx[1] * (Az[ijpk] - Az[I]) - b.idx[2] * (Ay[ijkp] - Ay[I]);
  if (in_j && i <= ng + b.n[0] && k <= ng + b.n[2])
    a.dBstag[1][I] = b.idx[2] * (Ax[ijkp] - Ax[I]) - b.idx[0] * (Az[ipjk] - Az[I]);
  if (in_k && i <= ng + b.n[0] && j <= ng + b.n[1])
    a.dBstag[2][I] = b.idx[0] * (Ay[ipjk] - Ay[I]) - b.idx[1] * (Ax[ijpk] - Ax[I]);
}
__global__ void __launch_bounds__(128)
    k_bstag(const C2PBoxArgs a) {
  bstag_body(a, blockIdx);
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
enum { C2P_FULL = 0, C2P_FAST = 1 };
template <class EOS, int MODE>
AXB_D bool c2p_cell(const C2PBoxArgs &a, const EOS &eos, const int i, const int j,
                    const int k, int &iters_first, bool &failed) {
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
    if constexpr (MODE == C2P_FAST) {
      if (mask_local != 1.0)
        return true;
    }
    if (MODE == C2P_FULL && a.excise && mask_local != 1.0) {
      seeds.entropy = eos.kappa_from_valid_rho_eps_ye(seeds.rho, seeds.eps, seeds.Ye);
      bh_interior<false>(eos, a.cp, atmo, seeds, cv, glo);
      pv = seeds;
      call_c2p = false;
    }
    cons_floors(cv, glo);
    if constexpr (MODE == C2P_FAST) {
      if (call_c2p) {
        Report r1;
        code = AXB_C2P_PRIME;
        palenzuela_solve<EOS, true>(eos, a.cp, atmo, pv, cv, glo, r1);
        if (r1.failed())
          return true; // REP_DEFER: every failure goes to the full cascade
        iters_first = r1.iters;
      }
    } else if (call_c2p) {
      Report r1, r2;
      code = AXB_C2P_PRIME;
      run_solver(a.c2p_prime, eos, a, atmo, pv, seeds, cv, glo, r1);
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
  return false;
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

template <class EOS>
AXB_D void c2p_box_body(const C2PBoxArgs &a, const EOS &eos, const uint3 bid) {
  __shared__ unsigned int s_hist[64];
  c2p_hist_init(a, s_hist);
  int i, j;
  const int k = a.b.ng + bid.z;
  const bool in_range = a.b.row_ij(a.b.ng, a.b.n[0], a.b.ng, a.b.n[1], bid, i, j);
  int iters_first = -1;
  bool failed = false;
  if (in_range)
    c2p_cell<EOS, C2P_FULL>(a, eos, i, j, k, iters_first, failed);
  c2p_epilogue(a, s_hist, iters_first, failed);
}
template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_MINB)
    k_c2p_box(const C2PBoxArgs a, const EOS eos) {
  c2p_box_body<EOS>(a, eos, blockIdx);
}

// Deferred cells of a fast pass: the count, then one entry per cell,
// i | j << 15 | k << 30 | box << 45 (box 0 for a single box).
struct C2PQueue {
  unsigned long long *count;
  unsigned long long *cell;
};
constexpr int C2P_QUEUE_MAX_EXTENT = 1 << 15; // per axis, ghosts included
constexpr int C2P_QUEUE_MAX_BOXES = 1 << 19;

// Fast pass over one tile: the common path, deferred cells appended to the
// queue (warp-aggregated).
template <class EOS>
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
    defer = c2p_cell<EOS, C2P_FAST>(a, eos, i, j, k, iters_first, failed);
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
  c2p_epilogue(a, s_hist, iters_first, failed);
}

// The full cascade over the queued cells; `args_of(box)` gives the box's
// argument block.  Every thread runs the same number of rounds, so the
// warp-level epilogue sees full warps.
template <class EOS, class ArgsOf>
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
      c2p_cell<EOS, C2P_FULL>(args_of(int(v >> 45)), eos, i, j, k, iters_first, failed);
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

template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_FAST_MINB)
    k_c2p_fast(const C2PBoxArgs a, const EOS eos, const C2PQueue q) {
  c2p_fast_body<EOS>(a, eos, blockIdx, 0, q);
}

template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_MINB)
    k_c2p_deferred(const C2PBoxArgs a, const EOS eos, const C2PQueue q) {
  c2p_deferred_body([&](int) -> const C2PBoxArgs & { return a; }, eos, q);
}

// whether a box's extent fits the queue's packing
inline bool c2p_queue_fits(const axb_box &b) {
  for (int d = 0; d < 3; ++d)
    if (b.n[d] + 2 * b.ng + 1 > C2P_QUEUE_MAX_EXTENT)
      return false;
  return true;
}
} // namespace axb

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

int check_box_c2p(const axb_box *b) {
  if (!b)
    return AXB_ERR_ARG;
  for (int d = 0; d < 3; ++d)
    if (b->n[d] < 1 || !(b->dx[d] > 0))
      return AXB_ERR_ARG;
  if (b->ng < 1)
    return AXB_ERR_GHOSTS;
  if (b->sy < b->n[0] + 2 * b->ng + 1 || b->sz < b->sy * (b->n[1] + 2 * b->ng + 1))
    return AXB_ERR_ARG;
  return AXB_OK;
}

C2PParams make_c2p_params(const axb_params &p) {
  C2PParams c;
  c.maxIter = p.max_iter;
  c.tol = p.c2p_tol;
  // c2p_1DPalenzuela.hxx:388-390, evaluated with the host libm like the
  // reference CPU build
  c.minbits = int(std::abs(std::log(p.c2p_tol)) / std::log(2.0));
  c.tolerance_0 = std::ldexp(1.0, -c.minbits);
  c.alp_thresh = p.alp_thresh;
  c.cons_error = p.cons_error_limit;
  c.vw_lim = p.vw_lim;
  c.w_lim = std::sqrt(1.0 + p.vw_lim * p.vw_lim);
  c.v_lim = p.vw_lim / c.w_lim;
  c.Bsq_lim = p.B_lim * p.B_lim;
  c.rho_BH = p.rho_BH;
  c.eps_BH = p.eps_BH;
  c.vwlim_BH = p.vwlim_BH;
  c.ye_lenient = p.Ye_lenient;
  c.use_zprim = p.use_z;
  c.use_temp = p.use_temperature;
  c.use_press_atmo = p.use_press_atmo;
  return c;
}

#define GFP(name) (f->gf[AXB_GF_##name])

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

int fill_c2p_args(axb_ctx *c, const axb_box *box, const axb_fields *f,
                  const axb_params *p, const axb_eos *eos, C2PBoxArgs &a) {
  int rc = check_box_c2p(box);
  if (rc)
    return rc;
  if (!f || !p || !eos)
    return AXB_ERR_ARG;
  const bool ok_solver = [](int s) {
    return s == AXB_C2P_NOBLE || s == AXB_C2P_PALENZUELA || s == AXB_C2P_ENTROPY;
  }(p->c2p_prime);
  if (!ok_solver || p->use_mask ||
      !(p->c2p_second == AXB_C2P_NOBLE || p->c2p_second == AXB_C2P_PALENZUELA ||
        p->c2p_second == AXB_C2P_ENTROPY || p->c2p_second == AXB_C2P_NONE))
    return AXB_ERR_UNSUPPORTED;
  // the entropy scheme needs p(rho, kappa), which a table does not define
  // (eos_3p_tabulated3d.hxx:315-333)
  const bool entropy = p->use_entropy_fix || p->c2p_prime == AXB_C2P_ENTROPY ||
                       p->c2p_second == AXB_C2P_ENTROPY;
  if (entropy && eos->kind != 0)
    return AXB_ERR_UNSUPPORTED;
  if (!(p->c2p_tol > 0) || p->max_iter < 1)
    return AXB_ERR_ARG;
  a.b = make_box(*box);
  a.Avec[0] = GFP(Avec_x);
  a.Avec[1] = GFP(Avec_y);
  a.Avec[2] = GFP(Avec_z);
  a.dBstag[0] = GFP(dBx_stag);
  a.dBstag[1] = GFP(dBy_stag);
  a.dBstag[2] = GFP(dBz_stag);
  a.alp = GFP(alp);
  const int gid[6] = {AXB_GF_gxx, AXB_GF_gxy, AXB_GF_gxz, AXB_GF_gyy, AXB_GF_gyz, AXB_GF_gzz};
  for (int q = 0; q < 6; ++q)
    a.g[q] = f->gf[gid[q]];
  a.dens = GFP(dens);
  a.mom[0] = GFP(momx);
  a.mom[1] = GFP(momy);
  a.mom[2] = GFP(momz);
  a.tau = GFP(tau);
  a.DYe = GFP(DYe);
  a.DEnt = GFP(DEnt);
  a.dB[0] = GFP(dBx);
  a.dB[1] = GFP(dBy);
  a.dB[2] = GFP(dBz);
  a.rho = GFP(rho);
  a.vel[0] = GFP(velx);
  a.vel[1] = GFP(vely);
  a.vel[2] = GFP(velz);
  a.eps = GFP(eps);
  a.press = GFP(press);
  a.temperature = GFP(temperature);
  a.Ye = GFP(Ye);
  a.entropy = GFP(entropy);
  a.Bvec[0] = GFP(Bvecx);
  a.Bvec[1] = GFP(Bvecy);
  a.Bvec[2] = GFP(Bvecz);
  a.saved_rho = GFP(saved_rho);
  a.saved_vel[0] = GFP(saved_velx);
  a.saved_vel[1] = GFP(saved_vely);
  a.saved_vel[2] = GFP(saved_velz);
  a.saved_eps = GFP(saved_eps);
  a.saved_Ye = GFP(saved_Ye);
  a.zvec[0] = GFP(zvec_x);
  a.zvec[1] = GFP(zvec_y);
  a.zvec[2] = GFP(zvec_z);
  a.svec[0] = GFP(svec_x);
  a.svec[1] = GFP(svec_y);
  a.svec[2] = GFP(svec_z);
  a.flag = GFP(con2prim_flag);
  const void *req[] = {a.Avec[0], a.Avec[1], a.Avec[2], a.dBstag[0], a.dBstag[1],
                       a.dBstag[2], a.alp, a.dens, a.mom[0], a.mom[1], a.mom[2],
                       a.tau, a.DYe, a.DEnt, a.rho, a.vel[0], a.vel[1], a.vel[2],
                       a.eps, a.press, a.temperature, a.Ye, a.entropy, a.Bvec[0],
                       a.Bvec[1], a.Bvec[2], a.saved_rho, a.saved_vel[0],
                       a.saved_vel[1], a.saved_vel[2], a.saved_eps, a.saved_Ye,
                       a.flag};
  for (const void *q : req)
    if (!q)
      return AXB_ERR_ARG;
  for (int q = 0; q < 6; ++q)
    if (!a.g[q])
      return AXB_ERR_ARG;
  a.cp = make_c2p_params(*p);
  a.c2p_prime = p->c2p_prime;
  a.c2p_second = p->c2p_second;
  a.use_entropy_fix = p->use_entropy_fix;
  a.excise = p->excise;
  a.thermal_eos_atmo = p->thermal_eos_atmo;
  a.use_press_atmo = p->use_press_atmo;
  a.rho_abs_min = p->rho_abs_min;
  a.r_atmo = p->r_atmo;
  a.n_rho_atmo = p->n_rho_atmo;
  a.p_atmo = p->p_atmo;
  a.n_press_atmo = p->n_press_atmo;
  a.t_atmo = p->t_atmo;
  a.n_temp_atmo = p->n_temp_atmo;
  a.Ye_atmo = p->Ye_atmo;
  a.atmo_tol = p->atmo_tol;
  a.poly = eos->poly;
  a.want_hist = 1;
  a.status = c->status;
  // the atmosphere is uniform when no cell lies beyond r_atmo
  double rmax2 = 0;
  for (int d = 0; d < 3; ++d) {
    const double lo = box->xmin[d], hi = box->xmin[d] + box->n[d] * box->dx[d];
    const double m = std::fmax(std::fabs(lo), std::fabs(hi));
    rmax2 += m * m;
  }
  a.atmo_uniform = std::sqrt(rmax2) <= p->r_atmo;
  if (eos->kind == 0) {
    a.gamma_noble = eos->ideal.gamma;
    a.Zmin = eos->ideal.rgrho.min;
    if (a.atmo_uniform)
      a.atmo_const = host_atmosphere(a, eos->ideal);
  } else if (eos->kind == 1) {
    // no eps(rho, press) for the tabulated EOS (the reference asserts,
    // eos_3p_tabulated3d.hxx:259-269): refuse the settings that need it
    // on every cell
    if (p->thermal_eos_atmo && p->use_press_atmo)
      return AXB_ERR_UNSUPPORTED;
    // the reader never sets the tabulated EOS's gamma, which the Noble
    // scheme reads (c2p_2DNoble.hxx); NaN makes that scheme fail cleanly
    a.gamma_noble = std::numeric_limits<double>::quiet_NaN();
    a.Zmin = eos->tab_h.rgrho.min;
    if (a.atmo_uniform)
      a.atmo_const = host_atmosphere(a, eos->tab_h);
  } else {
    return AXB_ERR_UNSUPPORTED;
  }
  return AXB_OK;
}

} // namespace

// ---------------------------------------------------------------------------
// batched forms (see axb_batch.cuh)
// ---------------------------------------------------------------------------
namespace {
__global__ void __launch_bounds__(128) k_bstag_batch(const C2PBoxArgs *args, const TileTable t, unsigned long long *ctr) {
  batch_loop(args, t, ctr, [&](const C2PBoxArgs &a, const uint3 bid) { bstag_body(a, bid); });
}
template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_MINB)
    k_c2p_box_batch(const C2PBoxArgs *args, const TileTable t, unsigned long long *ctr, const EOS eos) {
  batch_loop(args, t, ctr, [&](const C2PBoxArgs &a, const uint3 bid) {
    c2p_box_body<EOS>(a, eos, bid);
  });
}
template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_FAST_MINB)
    k_c2p_fast_batch(const C2PBoxArgs *args, const TileTable t, unsigned long long *ctr,
                     const EOS eos, const C2PQueue q) {
  batch_loop(args, t, ctr, [&](const C2PBoxArgs &a, const uint3 bid, int box) {
    c2p_fast_body<EOS>(a, eos, bid, box, q);
  });
}
template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_MINB)
    k_c2p_deferred_batch(const C2PBoxArgs *args, const EOS eos, const C2PQueue q) {
  c2p_deferred_body([&](int box) -> const C2PBoxArgs & { return args[box]; }, eos, q);
}
template <class EOS>
int launch_c2p_batch_eos(const C2PBoxArgs *a, const TileTable &t, unsigned long long *ctr,
                         const EOS &eos, int nblocks, unsigned long long *queue,
                         int deferred_blocks, cudaStream_t s) {
  if (!queue) {
    k_c2p_box_batch<<<nblocks, 128, 0, s>>>(a, t, ctr, eos);
  } else {
    C2PQueue q;
    q.count = queue;
    q.cell = queue + 1;
    if (cudaMemsetAsync(q.count, 0, sizeof(unsigned long long), s) != cudaSuccess)
      return AXB_ERR_CUDA;
    k_c2p_fast_batch<<<nblocks, 128, 0, s>>>(a, t, ctr, eos, q);
    k_c2p_deferred_batch<<<deferred_blocks, 128, 0, s>>>(a, eos, q);
  }
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}
} // namespace

namespace axb {
// The per-box post-step argument blocks of a batch (checked as
// axb_con2prim_group checks them), in device memory.
int batch_c2p_setup(axb_ctx *c, int nbox, const axb_box *boxes, const axb_fields *f,
                    const axb_params *p, const axb_eos *eos, void **out) {
  *out = nullptr;
  C2PBoxArgs *h = new (std::nothrow) C2PBoxArgs[nbox];
  if (!h)
    return AXB_ERR_ARG;
  for (int b = 0; b < nbox; ++b) {
    const int rc = fill_c2p_args(c, boxes + b, f + b, p, eos, h[b]);
    h[b].b.packed = 1;
    if (rc) {
      delete[] h;
      return rc;
    }
  }
  int rc = AXB_OK;
  if (cudaMalloc(out, nbox * sizeof(C2PBoxArgs)) != cudaSuccess ||
      cudaMemcpy(*out, h, nbox * sizeof(C2PBoxArgs), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = AXB_ERR_CUDA;
  delete[] h;
  return rc;
}

// batched grids over packed (i, j) planes: face curl (0), recovery (1)
uint3 c2p_grid(int which, const axb_box &b) {
  const int T = 128;
  const int e = which == 0 ? 2 : 0;
  const long long plane = (long long)(b.n[0] + e) * (b.n[1] + e);
  return make_uint3(unsigned((plane + T - 1) / T), 1, b.n[2] + e);
}

// `queue` (count, then room for every interior cell of the batch) selects
// the fast pass + deferred full cascade (Palenzuela first), else the full
// cascade in one launch.
int launch_c2p_batch(int which, const void *args, const TileTable &t,
                     unsigned long long *ctr, const axb_eos &eos, DevStatus *status,
                     int nblocks, cudaStream_t s, unsigned long long *queue,
                     int deferred_blocks) {
  if (t.total == 0)
    return AXB_OK;
  const C2PBoxArgs *a = static_cast<const C2PBoxArgs *>(args);
  if (which == 0) {
    k_bstag_batch<<<nblocks, 128, 0, s>>>(a, t, ctr);
    return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
  }
  if (eos.kind == 1)
    return launch_c2p_batch_eos(a, t, ctr, tab_for_launch(eos, status), nblocks, queue,
                                deferred_blocks, s);
  return launch_c2p_batch_eos(a, t, ctr, eos.ideal, nblocks, queue, deferred_blocks, s);
}

// whether a batch can take the fast pass: Palenzuela first, boxes and
// extents within the queue's packing
bool c2p_batch_fast_ok(int nbox, const axb_box *boxes, const axb_params *p) {
  if (p->c2p_prime != AXB_C2P_PALENZUELA || nbox > C2P_QUEUE_MAX_BOXES)
    return false;
  for (int b = 0; b < nbox; ++b)
    if (!c2p_queue_fits(boxes[b]))
      return false;
  return true;
}
} // namespace axb

// AsterX_Con2PrimGroup on one box (AsterX/schedule.ccl:119-165): replaces
// AsterX_ComputedBstagFromA (computeBfromA.cxx:58-65),
// AsterX_ComputedBFromdBstag (computeBfromA.cxx:67-85) and AsterX_Con2Prim
// (con2prim.cxx:457-502).
AXB_API int axb_con2prim_group(axb_ctx *c, const axb_box *box,
                               const axb_fields *f, const axb_params *p,
                               const axb_eos *eos, void *stream) {
  if (!c)
    return AXB_ERR_ARG;
  C2PBoxArgs a;
  int rc = fill_c2p_args(c, box, f, p, eos, a);
  if (rc)
    return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const BoxDev &b = a.b;
  const int T = 128;
  {
    // the (i, j) plane walked row after row (rows of n+2 faces)
    C2PBoxArgs ap = a;
    ap.b.packed = 1;
    const long long plane = (long long)(b.n[0] + 2) * (b.n[1] + 2);
    const dim3 grid(unsigned((plane + T - 1) / T), 1, b.n[2] + 2);
    axb_mark(c, AXB_R_BSTAG, s, true);
    k_bstag<<<grid, T, 0, s>>>(ap);
    axb_mark(c, AXB_R_BSTAG, s, false);
  }
  {
    const dim3 grid((b.n[0] + T - 1) / T, b.n[1], b.n[2]);
    axb_mark(c, AXB_R_C2P, s, true);
    if (a.c2p_prime == AXB_C2P_PALENZUELA && c2p_queue_fits(*box)) {
      // fast pass + the full cascade on the deferred cells; the queue (all
      // interior cells at most) comes from the stream-ordered allocator
      const unsigned long long ncell = (unsigned long long)b.n[0] * b.n[1] * b.n[2];
      void *buf = nullptr;
      if (axb_scratch_alloc(c, &buf, (ncell + 1) * sizeof(unsigned long long), s) !=
          cudaSuccess)
        return AXB_ERR_CUDA;
      C2PQueue q;
      q.count = static_cast<unsigned long long *>(buf);
      q.cell = q.count + 1;
      cudaMemsetAsync(q.count, 0, sizeof(unsigned long long), s);
      int sms = 148;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
      if (eos->kind == 1) {
        const EosTab t = tab_for_launch(*eos, a.status);
        k_c2p_fast<<<grid, T, 0, s>>>(a, t, q);
        k_c2p_deferred<<<4 * sms, T, 0, s>>>(a, t, q);
      } else {
        k_c2p_fast<<<grid, T, 0, s>>>(a, eos->ideal, q);
        k_c2p_deferred<<<4 * sms, T, 0, s>>>(a, eos->ideal, q);
      }
      cudaFreeAsync(buf, s);
    } else if (eos->kind == 1) {
      k_c2p_box<<<grid, T, 0, s>>>(a, tab_for_launch(*eos, a.status));
    } else {
      k_c2p_box<<<grid, T, 0, s>>>(a, eos->ideal);
    }
    axb_mark(c, AXB_R_C2P, s, false);
  }
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Independent-cell recovery (the per-cell body of AsterX_Con2Prim_typeEoS,
// con2prim.cxx:137-416, without grid, mask or graded atmosphere), with the
// optional learned initial guess.
// ---------------------------------------------------------------------------
namespace axb {
MlpDev mlp_device_view(const axb_mlp *m);
int mlp_nf(const axb_mlp *m);
int launch_mlp_guess(const axb_cells &c, const axb_mlp *m, float2 *guess, cudaStream_t s);

struct C2PCellsArgs {
  axb_cells c;
  C2PParams cp;
  int c2p_prime, c2p_second, use_entropy_fix;
  Atmo atmo;
  double gamma_noble, Zmin;
  int use_mlp;
  double bracket;
  MlpDev mlp;
  DevStatus *status;
};

template <class EOS>
AXB_D void run_solver_cells(int which, const EOS &eos, const C2PCellsArgs &a, Prim &pv,
                            Prim &seeds, Cons &cv, const sym3 &glo, Report &rep,
                            double zguess, double vsqguess, double xlo, double xhi) {
  if (which == AXB_C2P_NOBLE)
    noble_solve(eos, a.cp, a.atmo, a.gamma_noble, a.Zmin, pv, seeds, cv, glo, rep, zguess,
                vsqguess);
  else if (which == AXB_C2P_PALENZUELA)
    palenzuela_solve(eos, a.cp, a.atmo, pv, cv, glo, rep, xlo, xhi);
  else if (which == AXB_C2P_ENTROPY)
    entropy_solve(eos, a.cp, a.atmo, pv, cv, glo, rep);
}

template <class EOS>
__global__ void __launch_bounds__(128, AXB_C2P_MINB)
    k_c2p_cells(const C2PCellsArgs a, const EOS eos) {
  __shared__ unsigned int s_hist[64];
  for (int q = threadIdx.x; q < 64; q += blockDim.x)
    s_hist[q] = 0;
  __syncthreads();
  const axb_cells &c = a.c;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < c.n;
  Cons cv;
  sym3 glo{1, 0, 0, 1, 0, 1};
  if (valid) {
    cv.dens = c.dens[i];
    for (int q = 0; q < 3; ++q) {
      cv.mom[q] = c.mom[q][i];
      cv.dBvec[q] = c.dB[q][i];
    }
    cv.tau = c.tau[i];
    cv.DYe = c.DYe[i];
    cv.DEnt = c.DEnt ? c.DEnt[i] : 0.0;
    glo = sym3{c.g[0][i], c.g[1][i], c.g[2][i], c.g[3][i], c.g[4][i], c.g[5][i]};
  }
  // learned guess (x = h W, W) from k_mlp_guess
  double zguess = -1.0, vsqguess = -1.0, xlo = -1.0, xhi = -1.0;
  if (a.use_mlp && valid) {
    const float2 gs = reinterpret_cast<const float2 *>(c.guess)[i];
    const double x = gs.x, W = gs.y;
    zguess = cv.dens / sqrt(det3(glo)) * x; // Z = rho h W^2 = D (h W)
    vsqguess = 1.0 - 1.0 / (W * W);
    xlo = x * (1.0 - a.bracket);
    xhi = x * (1.0 + a.bracket);
    if (!(zguess > 0.0 && zguess < 1e300 && vsqguess >= 0.0 && vsqguess < 1.0))
      zguess = vsqguess = xlo = xhi = -1.0;
  }
  int iters_first = -1;
  bool failed = false, fallback = false;
  if (valid) {
    const double sqrt_detg = sqrt(det3(glo));
    const double isg = 1.0 / sqrt_detg;
    const double Bup[3] = {cv.dBvec[0] * isg, cv.dBvec[1] * isg, cv.dBvec[2] * isg};
    Prim pv;
    pv.set_nan();
    Prim seeds;
    if (c.seed_rho) {
      seeds.rho = c.seed_rho[i];
      seeds.eps = c.seed_eps[i];
      seeds.Ye = c.seed_Ye[i];
      for (int q = 0; q < 3; ++q)
        seeds.vel[q] = c.seed_vel[q][i];
      seeds.temperature = c.seed_temperature ? c.seed_temperature[i] : a.atmo.temp;
    } else { // cold start
      seeds.rho = cv.dens / sqrt_detg;
      seeds.eps = a.atmo.eps;
      seeds.Ye = cv.DYe / cv.dens;
      for (int q = 0; q < 3; ++q)
        seeds.vel[q] = 0.0;
      seeds.temperature = a.atmo.temp;
    }
    // the seed velocity is limited as in con2prim.cxx:168-209
    double v_low[3];
    lower3(glo, seeds.vel, v_low);
    const double vsq = dot3(v_low, seeds.vel);
    double zsq;
    if (vsq >= 1.0) {
      const double wlim = sqrt(1.0 + a.cp.vw_lim * a.cp.vw_lim);
      const double vlim = a.cp.vw_lim / wlim;
      for (int q = 0; q < 3; ++q)
        seeds.vel[q] *= vlim / sqrt(vsq);
      zsq = a.cp.vw_lim * a.cp.vw_lim;
    } else {
      zsq = vsq / (1.0 - vsq);
    }
    {
      double e = seeds.eps;
      seeds.press = eos.press_from_valid_rho_eps_ye(seeds.rho, e, seeds.Ye);
    }
    seeds.entropy = 0.0;
    for (int q = 0; q < 3; ++q) {
      seeds.Bvec[q] = Bup[q];
      seeds.E[q] = 0.0;
    }
    seeds.w_lor = sqrt(1.0 + zsq);
    int code;
    if (cv.dens <= sqrt_detg * a.atmo.rho_cut) {
      for (int q = 0; q < 3; ++q)
        pv.Bvec[q] = Bup[q];
      a.atmo.set(pv, cv, glo);
      code = AXB_C2P_ATMO;
      cons_floors(cv, glo);
    } else {
      cons_floors(cv, glo);
      Report r1, r2;
      code = AXB_C2P_PRIME;
      const bool guessed = zguess >= 0.0;
      const Prim seeds_plain = seeds; // the first scheme may overwrite its seeds
      run_solver_cells(a.c2p_prime, eos, a, pv, seeds, cv, glo, r1, zguess, vsqguess, xlo,
                       xhi);
      iters_first = r1.iters;
      if (r1.failed() && guessed) {
        // the guess led the first scheme astray: the plain cold start
        // (c2p_2DNoble.hxx:374-393, the plain bracket), then the plain cascade
        fallback = true;
        seeds = seeds_plain;
        pv.set_nan();
        Report rr;
        run_solver_cells(a.c2p_prime, eos, a, pv, seeds, cv, glo, rr, -1.0, -1.0, -1.0, -1.0);
        iters_first += rr.iters;
        r1 = rr;
      }
      if (r1.failed()) {
        code = AXB_C2P_SECOND;
        run_solver_cells(a.c2p_second, eos, a, pv, seeds, cv, glo, r2, -1.0, -1.0, -1.0,
                         -1.0);
      }
      bool recovered = false;
      if (r1.failed() && r2.failed() && a.use_entropy_fix) {
        Report re;
        entropy_solve(eos, a.cp, a.atmo, pv, cv, glo, re);
        recovered = !re.failed();
        if (recovered)
          code = AXB_C2P_ENTROPY_OK;
      }
      if (r1.failed() && r2.failed() && !recovered) {
        code = AXB_C2P_FAIL;
        failed = true;
        for (int q = 0; q < 3; ++q) {
          cv.dBvec[q] = sqrt_detg * Bup[q];
          pv.Bvec[q] = Bup[q];
        }
        a.atmo.set(pv, cv, glo);
      }
    }
    if (c.flag)
      c.flag[i] = code;
    if (c.fallback)
      c.fallback[i] = fallback ? 1.0 : 0.0;
    if (c.iters)
      c.iters[i] = iters_first;
    if (c.rho)
      c.rho[i] = pv.rho;
    if (c.eps)
      c.eps[i] = pv.eps;
    if (c.press)
      c.press[i] = pv.press;
    for (int q = 0; q < 3; ++q)
      if (c.vel[q])
        c.vel[q][i] = pv.vel[q];
    if (c.w_lorentz)
      c.w_lorentz[i] = pv.w_lor;
    if (c.Ye)
      c.Ye[i] = pv.Ye;
    if (c.temperature)
      c.temperature[i] = pv.temperature;
    if (c.entropy)
      c.entropy[i] = pv.entropy;
  }
  const unsigned nfail = __popc(__ballot_sync(0xffffffffu, failed));
  if (nfail && (threadIdx.x % 32) == 0) {
    atomicAdd(&a.status->c2p_fail_count, nfail);
    atomicOr(&a.status->error_word, AXB_EW_C2P_FAIL);
  }
  if (iters_first >= 0)
    atomicAdd(&s_hist[min(iters_first, 63)], 1u);
  __syncthreads();
  for (int q = threadIdx.x; q < 64; q += blockDim.x)
    if (s_hist[q])
      atomicAdd(&a.status->c2p_iter_hist[q], (unsigned long long)s_hist[q]);
}
} // namespace axb

AXB_API int axb_c2p_cells(axb_ctx *ctx, const axb_cells *cells, const axb_params *p,
                          const axb_eos *eos, const axb_mlp *mlp, void *stream) {
  if (!ctx || !cells || !p || !eos || cells->n < 0)
    return AXB_ERR_ARG;
  if (!cells->dens || !cells->tau || !cells->DYe)
    return AXB_ERR_ARG;
  for (int q = 0; q < 3; ++q)
    if (!cells->mom[q] || !cells->dB[q])
      return AXB_ERR_ARG;
  for (int q = 0; q < 6; ++q)
    if (!cells->g[q])
      return AXB_ERR_ARG;
  if (cells->seed_rho && (!cells->seed_eps || !cells->seed_Ye || !cells->seed_vel[0] ||
                          !cells->seed_vel[1] || !cells->seed_vel[2]))
    return AXB_ERR_ARG;
  auto ok_solver = [](int s) {
    return s == AXB_C2P_NOBLE || s == AXB_C2P_PALENZUELA || s == AXB_C2P_ENTROPY;
  };
  if (!ok_solver(p->c2p_prime) || !(ok_solver(p->c2p_second) || p->c2p_second == AXB_C2P_NONE))
    return AXB_ERR_UNSUPPORTED;
  const bool entropy = p->use_entropy_fix || p->c2p_prime == AXB_C2P_ENTROPY ||
                       p->c2p_second == AXB_C2P_ENTROPY;
  if (entropy && eos->kind != 0)
    return AXB_ERR_UNSUPPORTED; // p(rho, kappa) is not defined for a table
  if (entropy && !cells->DEnt)
    return AXB_ERR_ARG; // the entropy scheme reads the conserved entropy
  if (!(p->c2p_tol > 0) || p->max_iter < 1)
    return AXB_ERR_ARG;
  C2PCellsArgs a;
  a.c = *cells;
  a.cp = make_c2p_params(*p);
  a.c2p_prime = p->c2p_prime;
  a.c2p_second = p->c2p_second;
  a.use_entropy_fix = p->use_entropy_fix;
  a.status = ctx->status;
  a.use_mlp = mlp != nullptr;
  a.bracket = 0.0;
  if (mlp) {
    if (!cells->guess)
      return AXB_ERR_ARG;
    a.mlp = mlp_device_view(mlp);
    a.bracket = a.mlp.bracket;
    if (eos->kind == 1 && mlp_nf(mlp) != 9)
      return AXB_ERR_ARG; // the tabulated guess takes Ye as a ninth input
  }
  // uniform atmosphere as for a box inside r_atmo (host_atmosphere)
  C2PBoxArgs hb{};
  hb.thermal_eos_atmo = p->thermal_eos_atmo;
  hb.use_press_atmo = p->use_press_atmo;
  hb.rho_abs_min = p->rho_abs_min;
  hb.p_atmo = p->p_atmo;
  hb.t_atmo = p->t_atmo;
  hb.Ye_atmo = p->Ye_atmo;
  hb.atmo_tol = p->atmo_tol;
  hb.poly = eos->poly;
  if (eos->kind == 0) {
    a.gamma_noble = eos->ideal.gamma;
    a.Zmin = eos->ideal.rgrho.min;
    a.atmo = host_atmosphere(hb, eos->ideal);
  } else if (eos->kind == 1) {
    if (p->thermal_eos_atmo && p->use_press_atmo)
      return AXB_ERR_UNSUPPORTED;
    a.gamma_noble = std::numeric_limits<double>::quiet_NaN();
    a.Zmin = eos->tab_h.rgrho.min;
    a.atmo = host_atmosphere(hb, eos->tab_h);
  } else {
    return AXB_ERR_UNSUPPORTED;
  }
  if (cells->n == 0)
    return AXB_OK;
  const long long blocks = (cells->n + 127) / 128;
  if (blocks > 0x7fffffffLL)
    return AXB_ERR_TOO_LARGE;
  cudaStream_t s = (cudaStream_t)stream;
  if (mlp) {
    axb_mark(ctx, AXB_R_MLP, s, true);
    const int rc = launch_mlp_guess(*cells, mlp, reinterpret_cast<float2 *>(cells->guess), s);
    axb_mark(ctx, AXB_R_MLP, s, false);
    if (rc)
      return rc;
  }
  axb_mark(ctx, AXB_R_C2P_CELLS, s, true);
  if (eos->kind == 1)
    k_c2p_cells<<<(unsigned)blocks, 128, 0, s>>>(a, tab_for_launch(*eos, a.status));
  else
    k_c2p_cells<<<(unsigned)blocks, 128, 0, s>>>(a, eos->ideal);
  axb_mark(ctx, AXB_R_C2P_CELLS, s, false);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}
