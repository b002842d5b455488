// PostStep group of one box (AsterX_Con2PrimGroup, AsterX/schedule.ccl:
// 119-165): curl A -> dB_stag, face-to-cell dB, and the con2prim driver with
// its Noble -> Palenzuela -> atmosphere cascade (AsterX/src/con2prim.cxx:
// 73-454); the device code is in axb_c2p_box.cuh.
#include "axb_c2p_box.cuh"
#include "axb_mlp.cuh"

using namespace axb;

namespace axb {
__global__ void __launch_bounds__(128)
    k_bstag(const C2PBoxArgs a) {
  bstag_body(a, blockIdx);
}
} // namespace axb

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace axb {

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
  a.guess = nullptr;
  a.bracket = 0.0;
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
  // upwind CT reconstructs dB_stag to the edges from three faces out
  a.bext = p->use_uct ? 3 : 1;
  if (a.bext > box->ng)
    return AXB_ERR_GHOSTS;
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

} // namespace axb

namespace axb {
MlpDev mlp_device_view(const axb_mlp *m);
int mlp_nf(const axb_mlp *m);
int launch_mlp_guess_box(const MlpBoxIn &in, const axb_mlp *m, float2 *guess,
                         DevStatus *status, cudaStream_t s);

// the recovery kernels of one box, with or without the learned guess
template <bool GUESS>
void launch_box_recovery(const C2PBoxArgs &a, const axb_eos *eos, const dim3 grid, int T,
                         bool fast, const C2PQueue &q, int sms, cudaStream_t s) {
  if (fast) {
    if (eos->kind == 1) {
      const EosTab t = tab_for_launch(*eos, a.status);
      k_c2p_fast<EosTab, GUESS><<<grid, T, 0, s>>>(a, t, q);
      k_c2p_deferred<EosTab, GUESS><<<4 * sms, T, 0, s>>>(a, t, q);
    } else {
      k_c2p_fast<EosIdeal, GUESS><<<grid, T, 0, s>>>(a, eos->ideal, q);
      k_c2p_deferred<EosIdeal, GUESS><<<4 * sms, T, 0, s>>>(a, eos->ideal, q);
    }
  } else if (eos->kind == 1) {
    k_c2p_box<EosTab, GUESS><<<grid, T, 0, s>>>(a, tab_for_launch(*eos, a.status));
  } else {
    k_c2p_box<EosIdeal, GUESS><<<grid, T, 0, s>>>(a, eos->ideal);
  }
}

int con2prim_group_run(axb_ctx *c, const axb_box *box, const axb_fields *f,
                       const axb_params *p, const axb_eos *eos, const axb_mlp *mlp,
                       void *stream) {
  if (!c)
    return AXB_ERR_ARG;
  C2PBoxArgs a;
  int rc = fill_c2p_args(c, box, f, p, eos, a);
  if (rc)
    return rc;
  if (mlp && eos->kind == 1 && mlp_nf(mlp) != 9)
    return AXB_ERR_ARG; // the tabulated guess takes Ye as a ninth input
  cudaStream_t s = (cudaStream_t)stream;
  const BoxDev &b = a.b;
  const int T = 128;
  {
    // the (i, j) plane walked row after row (rows of n+2 faces)
    C2PBoxArgs ap = a;
    ap.b.packed = 1;
    const int e = a.bext;
    const long long plane = (long long)(b.n[0] + 2 * e) * (b.n[1] + 2 * e);
    const dim3 grid(unsigned((plane + T - 1) / T), 1, b.n[2] + 2 * e);
    axb_mark(c, AXB_R_BSTAG, s, true);
    k_bstag<<<grid, T, 0, s>>>(ap);
    axb_mark(c, AXB_R_BSTAG, s, false);
  }
  const unsigned long long ncell = (unsigned long long)b.n[0] * b.n[1] * b.n[2];
  void *gbuf = nullptr;
  if (mlp) {
    // the guess of every interior cell from its conserved variables, the
    // dB_stag just computed and the metric, ahead of the recovery
    if (axb_scratch_alloc(c, &gbuf, ncell * sizeof(float2), s) != cudaSuccess)
      return AXB_ERR_CUDA;
    MlpBoxIn in;
    in.b = a.b;
    in.dens = a.dens;
    in.tau = a.tau;
    in.DYe = a.DYe;
    for (int q = 0; q < 3; ++q) {
      in.mom[q] = a.mom[q];
      in.dBstag[q] = a.dBstag[q];
    }
    for (int q = 0; q < 6; ++q)
      in.g[q] = a.g[q];
    axb_mark(c, AXB_R_MLP, s, true);
    rc = launch_mlp_guess_box(in, mlp, static_cast<float2 *>(gbuf), a.status, s);
    axb_mark(c, AXB_R_MLP, s, false);
    if (rc) {
      cudaFreeAsync(gbuf, s);
      return rc;
    }
    a.guess = static_cast<const float2 *>(gbuf);
    a.bracket = mlp_device_view(mlp).bracket;
  }
  {
    const dim3 grid((b.n[0] + T - 1) / T, b.n[1], b.n[2]);
    axb_mark(c, AXB_R_C2P, s, true);
    const bool fast = a.c2p_prime == AXB_C2P_PALENZUELA && c2p_queue_fits(*box);
    void *buf = nullptr;
    C2PQueue q{nullptr, nullptr};
    int sms = 148;
    if (fast) {
      // fast pass + the full cascade on the deferred cells; the queue (all
      // interior cells at most) comes from the stream-ordered allocator
      if (axb_scratch_alloc(c, &buf, (ncell + 1) * sizeof(unsigned long long), s) !=
          cudaSuccess) {
        if (gbuf)
          cudaFreeAsync(gbuf, s);
        return AXB_ERR_CUDA;
      }
      q.count = static_cast<unsigned long long *>(buf);
      q.cell = q.count + 1;
      cudaMemsetAsync(q.count, 0, sizeof(unsigned long long), s);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    }
    if (mlp)
      launch_box_recovery<true>(a, eos, grid, T, fast, q, sms, s);
    else
      launch_box_recovery<false>(a, eos, grid, T, fast, q, sms, s);
    if (buf)
      cudaFreeAsync(buf, s);
    if (gbuf)
      cudaFreeAsync(gbuf, s);
    axb_mark(c, AXB_R_C2P, s, false);
  }
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}
} // namespace axb

// AsterX_Con2PrimGroup on one box (AsterX/schedule.ccl:119-165): replaces
// AsterX_ComputedBstagFromA (computeBfromA.cxx:58-65),
// AsterX_ComputedBFromdBstag (computeBfromA.cxx:67-85) and AsterX_Con2Prim
// (con2prim.cxx:457-502).
AXB_API int axb_con2prim_group(axb_ctx *c, const axb_box *box,
                               const axb_fields *f, const axb_params *p,
                               const axb_eos *eos, void *stream) {
  return con2prim_group_run(c, box, f, p, eos, nullptr, stream);
}

// The same with the learned initial guess of the first solver (no
// counterpart in the reference): Noble's seeds or Palenzuela's bracket from
// the network, a failed guessed attempt retried from the plain seeds.
AXB_API int axb_con2prim_group_guess(axb_ctx *c, const axb_box *box, const axb_fields *f,
                                     const axb_params *p, const axb_eos *eos,
                                     const axb_mlp *mlp, void *stream) {
  if (!mlp)
    return AXB_ERR_ARG;
  return con2prim_group_run(c, box, f, p, eos, mlp, stream);
}
