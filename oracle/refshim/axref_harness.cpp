// Test infrastructure only.  Drives the reference hot-path translation units
// (AsterX/src/{fluxes,source,rhs,computeBfromA,con2prim,tmunu}.cxx, compiled
// unmodified against the stand-in headers of this directory) and the
// reference per-point headers through a small C ABI, so that tests can
// compare the oracle restatement and the CUDA kernels with the reference's
// own code on the same inputs.  Built by oracle/build_oracle.py into
// oracle/_ref/libaxref.so.
#include <cstring>
#include <cctk.h>
#include <cctk_Arguments.h>
#include <cctk_Parameters.h>
#include <loop_device.hxx>

#include "c2p_1DPalenzuela.hxx"
#include "c2p_2DNoble.hxx"
#include "eigenvalues.hxx"
#include "fluxes.hxx"
#include "prim2con.hxx"
#include "reconstruct.hxx"
#include "setup_eos.hxx"

#include <sstream>
#include <vector>

#include "estimate_error.hxx"

#include "../../include/asterx_b200.h"

#include <cstdio>
#include <new>
#include <stdexcept>
#include <string>

#define ORA_API extern "C" __attribute__((visibility("default")))

// ---------------------------------------------------------------------------
// globals the reference code and the stand-in headers refer to
// ---------------------------------------------------------------------------
axref_params_t axref_params;

namespace EOSX {
eos_1p_polytropic *global_eos_1p_poly = nullptr;
eos_3p_idealgas *global_eos_3p_ig = nullptr;
eos_3p_hybrid *global_eos_3p_hyb = nullptr;
eos_3p_tabulated3d *global_eos_3p_tab3d = nullptr;
} // namespace EOSX

namespace AsterX {
extern "C" void AsterX_Fluxes(CCTK_ARGUMENTS);
extern "C" void AsterX_SourceTerms(CCTK_ARGUMENTS);
extern "C" void AsterX_RHS(CCTK_ARGUMENTS);
extern "C" void AsterX_ComputedBstagFromA(CCTK_ARGUMENTS);
extern "C" void AsterX_ComputedBFromdBstag(CCTK_ARGUMENTS);
extern "C" void AsterX_Con2Prim(CCTK_ARGUMENTS);
extern "C" void AsterX_Tmunu(CCTK_ARGUMENTS);
} // namespace AsterX

// The Cactus group tables that estimate_error.hxx's parameter parsing reads
// (never reached: the checker passes the regrid variables itself).
int CCTK_GroupTagsTableI(int) { axref_fatal("CCTK_GroupTagsTableI is not available"); }
int CCTK_GroupCenteringTableI(int) {
  axref_fatal("CCTK_GroupCenteringTableI is not available");
}
int Util_TableGetIntArray(int, int, int *, const char *) {
  axref_fatal("Util_TableGetIntArray is not available");
}

namespace {
double *g_fields[AXREF_NFIELDS];
Loop::GridDescBaseDevice g_grid;
long long g_sy = 0, g_sz = 0;
CCTK_REAL g_delta[3];
cGH g_gh{0};
const char *g_names[] = {
#define AXREF_NAME(name) #name,
    AXREF_FIELD_LIST(AXREF_NAME)
#undef AXREF_NAME
};
char g_errmsg[512] = "";

struct axref_abort : std::runtime_error {
  using std::runtime_error::runtime_error;
};

const char *recon_name(int r) {
  switch (r) {
  case AXB_RECON_GODUNOV: return "Godunov";
  case AXB_RECON_MINMOD: return "minmod";
  case AXB_RECON_MONOCENTRAL: return "monocentral";
  case AXB_RECON_PPM: return "ppm";
  case AXB_RECON_EPPM: return "eppm";
  case AXB_RECON_WENOZ: return "wenoz";
  case AXB_RECON_MP5: return "mp5";
  }
  return "invalid";
}
const char *c2p_name(int c) {
  switch (c) {
  case AXB_C2P_NONE: return "None";
  case AXB_C2P_NOBLE: return "Noble";
  case AXB_C2P_PALENZUELA: return "Palenzuela";
  case AXB_C2P_ENTROPY: return "Entropy";
  }
  return "invalid";
}

template <typename F> int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const axref_abort &e) {
    snprintf(g_errmsg, sizeof g_errmsg, "%s", e.what());
    return 1;
  }
}
} // namespace

[[noreturn]] void axref_fatal(const char *msg) { throw axref_abort(msg); }
double *axref_field(int id) { return g_fields[id]; }
long long axref_sy() { return g_sy; }
long long axref_sz() { return g_sz; }
const Loop::GridDescBaseDevice &axref_grid() { return g_grid; }
const CCTK_REAL *axref_delta_space() { return g_delta; }

ORA_API const char *ora_last_error() { return g_errmsg; }

ORA_API int ora_bind(const char *name, double *ptr) {
  for (int i = 0; i < AXREF_NFIELDS; ++i)
    if (std::strcmp(g_names[i], name) == 0) {
      g_fields[i] = ptr;
      return 0;
    }
  return 1; // names the reference does not know (engine scratch) are ignored
}

ORA_API int ora_setup(const axb_box *b, const axb_params *p, int iteration) {
  for (int d = 0; d < 3; ++d) {
    g_grid.nghostzones[d] = b->ng;
    g_grid.ncells[d] = b->n[d];
    g_grid.dx[d] = b->dx[d];
    g_grid.xmin[d] = b->xmin[d];
    g_delta[d] = b->dx[d];
  }
  g_grid.ext_c = g_grid.ext_v = 0;
  g_sy = b->sy;
  g_sz = b->sz;
  g_gh.iteration = iteration;

  axref_params_t &q = axref_params;
  q.recon_type = p->recon_type == AXB_RECVAR_V   ? "v_vec"
                 : p->recon_type == AXB_RECVAR_Z ? "z_vec"
                                                 : "s_vec";
  q.reconstruction_method = recon_name(p->reconstruction_method);
  q.loworder_method = recon_name(p->loworder_method);
  q.flux_type = p->flux_type == AXB_FLUX_HLLE ? "HLLE" : "LxF";
  q.vector_potential_gauge = p->vector_potential_gauge == AXB_GAUGE_ALGEBRAIC
                                 ? "algebraic"
                                 : "generalized Lorentz";
  q.c2p_prime = c2p_name(p->c2p_prime);
  q.c2p_second = c2p_name(p->c2p_second);
  q.reconstruct_with_temperature = p->reconstruct_with_temperature;
  q.ppm_shock_detection = p->ppm_shock_detection;
  q.ppm_zone_flattening = p->ppm_zone_flattening;
  q.use_uct = p->use_uct;
  q.local_spatial_order = p->local_spatial_order;
  q.thermal_eos_atmo = p->thermal_eos_atmo;
  q.use_press_atmo = p->use_press_atmo;
  q.max_iter = p->max_iter;
  q.use_mask = p->use_mask;
  q.excise = p->excise;
  q.debug_mode = 0;
  q.use_entropy_fix = p->use_entropy_fix;
  q.Ye_lenient = p->Ye_lenient;
  q.use_z = p->use_z;
  q.use_temperature = p->use_temperature;
  q.interpolate_failed_c2p = 0;
  q.poly_k = p->poly_k;
  q.poly_gamma = p->poly_gamma;
  q.ppm_eta1 = p->ppm_eta1;
  q.ppm_eta2 = p->ppm_eta2;
  q.ppm_eps = p->ppm_eps;
  q.ppm_eps_shock = p->ppm_eps_shock;
  q.ppm_small = p->ppm_small;
  q.ppm_omega1 = p->ppm_omega1;
  q.ppm_omega2 = p->ppm_omega2;
  q.enhanced_ppm_C2 = p->enhanced_ppm_C2;
  q.weno_eps = p->weno_eps;
  q.mp5_alpha = p->mp5_alpha;
  q.lorenz_damp_fac = p->lorenz_damp_fac;
  q.r_atmo = p->r_atmo;
  q.rho_abs_min = p->rho_abs_min;
  q.n_rho_atmo = p->n_rho_atmo;
  q.p_atmo = p->p_atmo;
  q.n_press_atmo = p->n_press_atmo;
  q.Ye_atmo = p->Ye_atmo;
  q.t_atmo = p->t_atmo;
  q.n_temp_atmo = p->n_temp_atmo;
  q.atmo_tol = p->atmo_tol;
  q.c2p_tol = p->c2p_tol;
  q.alp_thresh = p->alp_thresh;
  q.cons_error_limit = p->cons_error_limit;
  q.vw_lim = p->vw_lim;
  q.B_lim = p->B_lim;
  q.rho_BH = p->rho_BH;
  q.eps_BH = p->eps_BH;
  q.vwlim_BH = p->vwlim_BH;
  q.eps_atmo = p->eps_atmo;
  q.gl_gamma = 0; // only read by the out-of-scope interpolate-failed path
  return 0;
}

ORA_API void ora_set_ext(int ext_c, int ext_v) {
  g_grid.ext_c = ext_c;
  g_grid.ext_v = ext_v;
}

// Ideal-gas evolution EOS and the polytrope used for the cold atmosphere,
// built as EOSX_Setup_EOS / EOSX_Setup_EOSID do (EOSX/src/setup_eos.cxx:
// 24-78).
ORA_API int ora_eos_idealgas(double gamma, double umass, double rho_min,
                             double rho_max, double eps_min, double eps_max,
                             double ye_min, double ye_max, double poly_gamma,
                             double poly_k) {
  using namespace EOSX;
  return guarded([&] {
    static eos_3p_idealgas ig;
    static eos_1p_polytropic poly;
    new (&poly) eos_1p_polytropic;
    poly.init(poly_gamma, poly_k, rho_max);
    new (&ig) eos_3p_idealgas;
    eos_3p::range rgeps(eps_min, eps_max), rgrho(rho_min, rho_max),
        rgye(ye_min, ye_max);
    ig.init(gamma, umass, rgeps, rgrho, rgye);
    global_eos_3p_ig = &ig;
    global_eos_1p_poly = &poly;
    axref_params.evolution_eos = "IdealGas";
  });
}

// Tabulated3d EOS built in memory from an already-converted table (natural
// logs of rho and T, Ye, 19 variables interleaved variable-fastest as the
// reference's reader leaves them, eos_3p_tabulated3d.hxx:141-177), then the
// same range set-up as the end of eos_3p_tabulated3d::init (:179-192).
ORA_API int ora_eos_tabulated(int nrho, int ntemp, int nye,
                              const double *logrho, const double *logtemp,
                              const double *yes, const double *table,
                              double energy_shift, double poly_gamma,
                              double poly_k) {
  using namespace EOSX;
  return guarded([&] {
    static eos_3p_tabulated3d tab;
    static eos_1p_polytropic poly;
    static double shift;
    static linear_interp_uniform_ND_t<CCTK_REAL, 3, NTABLES> *interp = nullptr;
    new (&poly) eos_1p_polytropic;
    poly.init(poly_gamma, poly_k, 1.0);
    new (&tab) eos_3p_tabulated3d;
    shift = energy_shift;
    tab.energy_shift = &shift;
    tab.gamma = std::numeric_limits<double>::quiet_NaN(); // never set by init
    std::array<size_t, 3> dims{size_t(nrho), size_t(ntemp), size_t(nye)};
    interp = (decltype(interp))std::malloc(sizeof(*interp));
    new (interp) linear_interp_uniform_ND_t<CCTK_REAL, 3, NTABLES>(
        const_cast<double *>(table), dims, const_cast<double *>(logrho),
        const_cast<double *>(logtemp), const_cast<double *>(yes));
    tab.interptable = interp;
    tab.rgrho = eos_3p::range{exp(interp->xmin<0>()), exp(interp->xmax<0>())};
    tab.rgtemp = eos_3p::range{exp(interp->xmin<1>()), exp(interp->xmax<1>())};
    tab.rgye = eos_3p::range{interp->xmin<2>(), interp->xmax<2>()};
    tab.rgeps = tab.compute_eps_range_full_table();
    global_eos_3p_tab3d = &tab;
    global_eos_1p_poly = &poly;
    axref_params.evolution_eos = "Tabulated3d";
  });
}

// The reference's StellarCollapse reader (eos_3p_tabulated3d::init,
// EOSX/src/eos_3p_tabulated3d/eos_3p_tabulated3d.hxx:53-193) on datasets
// registered in memory (the stand-in HDF5 of refshim/hdf5.h): ora_h5_clear,
// ora_h5_put_* per dataset, then ora_eos_stellarcollapse, which makes the
// result the EOS of the following routines; ora_eos_tab_export copies its
// converted axes, table and energy shift out.
ORA_API void ora_h5_clear() {
  axref_h5_store().clear();
  axref_h5_handles().clear();
}
ORA_API void ora_h5_put_double(const char *name, const double *v, long n) {
  axref_h5_dset &d = axref_h5_store()[name];
  d.is_int = false;
  d.d.assign(v, v + n);
}
ORA_API void ora_h5_put_int(const char *name, const int *v, long n) {
  axref_h5_dset &d = axref_h5_store()[name];
  d.is_int = true;
  d.i.assign(v, v + n);
}
ORA_API int ora_eos_stellarcollapse(double poly_gamma, double poly_k) {
  using namespace EOSX;
  return guarded([&] {
    static eos_3p_tabulated3d tab;
    static eos_1p_polytropic poly;
    new (&poly) eos_1p_polytropic;
    poly.init(poly_gamma, poly_k, 1.0);
    new (&tab) eos_3p_tabulated3d;
    tab.gamma = std::numeric_limits<double>::quiet_NaN(); // never set by init
    eos_3p::range rgeps, rgrho, rgye;
    tab.init("in-memory", rgeps, rgrho, rgye);
    global_eos_3p_tab3d = &tab;
    global_eos_1p_poly = &poly;
    axref_params.evolution_eos = "Tabulated3d";
  });
}
ORA_API void ora_eos_tab_export(double *logrho, double *logtemp, double *ye, double *table,
                                double *energy_shift) {
  auto *t = EOSX::global_eos_3p_tab3d;
  auto *it = t->interptable;
  const size_t n0 = it->num_points[0], n1 = it->num_points[1], n2 = it->num_points[2];
  std::memcpy(logrho, it->x[0], n0 * sizeof(double));
  std::memcpy(logtemp, it->x[1], n1 * sizeof(double));
  std::memcpy(ye, it->x[2], n2 * sizeof(double));
  std::memcpy(table, it->y, n0 * n1 * n2 * NTABLES * sizeof(double));
  *energy_shift = *t->energy_shift;
}

ORA_API void ora_eos_tab_ranges(double *out8) {
  auto *t = EOSX::global_eos_3p_tab3d;
  out8[0] = t->rgrho.min, out8[1] = t->rgrho.max;
  out8[2] = t->rgtemp.min, out8[3] = t->rgtemp.max;
  out8[4] = t->rgye.min, out8[5] = t->rgye.max;
  out8[6] = t->rgeps.min, out8[7] = t->rgeps.max;
}

// ---------------------------------------------------------------------------
// scheduled routines
// ---------------------------------------------------------------------------
ORA_API int ora_fluxes() { return guarded([] { AsterX::AsterX_Fluxes(&g_gh); }); }
ORA_API int ora_sources() {
  return guarded([] { AsterX::AsterX_SourceTerms(&g_gh); });
}
ORA_API int ora_rhs() { return guarded([] { AsterX::AsterX_RHS(&g_gh); }); }
ORA_API int ora_bstag() {
  return guarded([] { AsterX::AsterX_ComputedBstagFromA(&g_gh); });
}
ORA_API int ora_dB() {
  return guarded([] { AsterX::AsterX_ComputedBFromdBstag(&g_gh); });
}
ORA_API int ora_c2p() { return guarded([] { AsterX::AsterX_Con2Prim(&g_gh); }); }

// ---------------------------------------------------------------------------
// per-point entry points
// ---------------------------------------------------------------------------
namespace {
ReconX::reconstruct_params_t recon_params() {
  ReconX::reconstruct_params_t r;
  const axref_params_t &q = axref_params;
  r.ppm_shock_detection = q.ppm_shock_detection;
  r.ppm_zone_flattening = q.ppm_zone_flattening;
  r.poly_k = q.poly_k;
  r.poly_gamma = q.poly_gamma;
  r.ppm_eta1 = q.ppm_eta1;
  r.ppm_eta2 = q.ppm_eta2;
  r.ppm_eps = q.ppm_eps;
  r.ppm_eps_shock = q.ppm_eps_shock;
  r.ppm_small = q.ppm_small;
  r.ppm_omega1 = q.ppm_omega1;
  r.ppm_omega2 = q.ppm_omega2;
  r.enhanced_ppm_C2 = q.enhanced_ppm_C2;
  r.weno_eps = q.weno_eps;
  r.mp5_alpha = q.mp5_alpha;
  return r;
}
} // namespace

// ReconX::reconstruct (ReconX/src/reconstruct.hxx:36-103) on a 6-cell
// pencil v[0..5] = Immm..Ippp, with press and the velocity along the pencil
// given on the same six cells.
ORA_API void ora_reconstruct(int method, const double *v, const double *pr,
                             const double *vel, int is_rho, int is_press,
                             double *out) {
  double bv[6], bp[6], bu[6];
  for (int i = 0; i < 6; ++i)
    bv[i] = v[i], bp[i] = pr[i], bu[i] = vel[i];
  const Loop::GF3D2<const double> gv(bv, 6, 6), gp(bp, 6, 6), gu(bu, 6, 6);
  Loop::PointDesc p;
  p.I = Arith::vect<int, 3>{3, 0, 0};
  for (int d = 0; d < 3; ++d)
    p.DI[d] = Arith::vect<int, 3>{d == 0, d == 1, d == 2};
  const auto rp = recon_params();
  const auto r = ReconX::reconstruct(gv, p, ReconX::reconstruction_t(method),
                                     0, bool(is_rho), bool(is_press), gp, gu,
                                     rp);
  out[0] = r[0];
  out[1] = r[1];
}

// AsterX::eigenvalues followed by laxf / hlle (AsterX/src/eigenvalues.hxx:
// 19-79, AsterX/src/fluxes.hxx:20-49).  in = alp, beta, u, then the pairs
// vel, rho, cs2, w, h, bsq; lam receives the 8 speeds.
ORA_API void ora_eigen(const double *in, double *lam) {
  using Arith::vec;
  const vec<double, 2> vel{in[3], in[4]}, rho{in[5], in[6]}, cs2{in[7], in[8]},
      w{in[9], in[10]}, h{in[11], in[12]}, bsq{in[13], in[14]};
  const auto l = AsterX::eigenvalues(in[0], in[1], in[2], vel, rho, cs2, w, h, bsq);
  for (int s = 0; s < 2; ++s)
    for (int i = 0; i < 4; ++i)
      lam[4 * s + i] = l(s)(i);
}
ORA_API double ora_riemann(int flux_type, const double *lam, double uL,
                           double uR, double fL, double fR) {
  using Arith::vec;
  const vec<vec<double, 4>, 2> L{vec<double, 4>{lam[0], lam[1], lam[2], lam[3]},
                                 vec<double, 4>{lam[4], lam[5], lam[6], lam[7]}};
  const vec<double, 2> u{uL, uR}, f{fL, fR};
  return flux_type == AXB_FLUX_HLLE ? AsterX::hlle(L, u, f) : AsterX::laxf(L, u, f);
}

// AsterX::prim2con (AsterX/src/prim2con.hxx:38-83).
// prim = rho, vx, vy, vz, eps, press, entropy, Ye, Bx, By, Bz;
// cons = dens, momx, momy, momz, tau, DEnt, DYe, dBx, dBy, dBz.
ORA_API void ora_prim2con(const double *g6, const double *prim, double *cons) {
  const Arith::smat<double, 3> g{g6[0], g6[1], g6[2], g6[3], g6[4], g6[5]};
  AsterX::prim pv;
  pv.rho = prim[0];
  pv.vel = Arith::vec<double, 3>{prim[1], prim[2], prim[3]};
  pv.eps = prim[4];
  pv.press = prim[5];
  pv.entropy = prim[6];
  pv.Ye = prim[7];
  pv.Bvec = Arith::vec<double, 3>{prim[8], prim[9], prim[10]};
  AsterX::cons cv;
  AsterX::prim2con(g, pv, cv);
  cons[0] = cv.dens;
  for (int i = 0; i < 3; ++i)
    cons[1 + i] = cv.mom(i), cons[7 + i] = cv.dBvec(i);
  cons[4] = cv.tau;
  cons[5] = cv.DEnt;
  cons[6] = cv.DYe;
}

// One Con2PrimFactory functor on one cell (c2p_2DNoble::solve,
// c2p_2DNoble.hxx:275-594, or c2p_1DPalenzuela::solve,
// c2p_1DPalenzuela.hxx:306-556) with an explicit atmosphere.
//   cons[10]  = dens, momx, momy, momz, tau, DYe, DEnt, dBx, dBy, dBz (in/out)
//   g6        = gxx, gxy, gxz, gyy, gyz, gzz
//   seed[9]   = rho, eps, Ye, press, temperature, entropy, vx, vy, vz (Noble)
//   atmo[7]   = rho, eps, Ye, press, temp, entropy, rho_cut
//   prim[16]  = rho, eps, Ye, press, temperature, entropy, vx, vy, vz, w_lor,
//               Bx, By, Bz, Ex, Ey, Ez
//   rep[3]    = status, iters, adjust_cons
template <typename EOS>
static void c2p_point_eos(const EOS *eos, int solver, double *cons,
                          const double *g6, const double *seed,
                          const double *atmo_in, double *prim, int *rep3) {
  using namespace Con2PrimFactory;
  const axref_params_t &q = axref_params;
  const atmosphere atmo(atmo_in[0], atmo_in[1], atmo_in[2], atmo_in[3],
                        atmo_in[4], atmo_in[5], atmo_in[6]);
  const Arith::smat<double, 3> glo{g6[0], g6[1], g6[2], g6[3], g6[4], g6[5]};
  cons_vars cv{cons[0], {cons[1], cons[2], cons[3]}, cons[4], cons[5],
               cons[6], {cons[7], cons[8], cons[9]}};
  prim_vars pv;
  pv.set_to_nan();
  c2p_report rep;
  if (solver == AXB_C2P_NOBLE) {
    const double sdetg = sqrt(Arith::calc_det(glo));
    const Arith::vec<double, 3> Bup{cv.dBvec(0) / sdetg, cv.dBvec(1) / sdetg,
                                    cv.dBvec(2) / sdetg};
    prim_vars seeds{seed[0], seed[1], seed[2], seed[3], seed[4], seed[5],
                    {seed[6], seed[7], seed[8]}, 1.0, Bup};
    c2p_2DNoble s(eos, atmo, q.max_iter, q.c2p_tol, q.alp_thresh,
                  q.cons_error_limit, q.vw_lim, q.B_lim, q.rho_BH, q.eps_BH,
                  q.vwlim_BH, q.Ye_lenient, q.use_z, q.use_temperature,
                  q.use_press_atmo);
    s.solve(eos, pv, seeds, cv, glo, rep);
  } else {
    c2p_1DPalenzuela s(eos, atmo, q.max_iter, q.c2p_tol, q.alp_thresh,
                       q.cons_error_limit, q.vw_lim, q.B_lim, q.rho_BH,
                       q.eps_BH, q.vwlim_BH, q.Ye_lenient, q.use_z,
                       q.use_temperature, q.use_press_atmo);
    s.solve(eos, pv, cv, glo, rep);
  }
  cons[0] = cv.dens;
  for (int i = 0; i < 3; ++i)
    cons[1 + i] = cv.mom(i), cons[7 + i] = cv.dBvec(i);
  cons[4] = cv.tau;
  cons[5] = cv.DYe;
  cons[6] = cv.DEnt;
  const double pvals[16] = {pv.rho,     pv.eps,     pv.Ye,      pv.press,
                            pv.temperature, pv.entropy, pv.vel(0), pv.vel(1),
                            pv.vel(2),  pv.w_lor,   pv.Bvec(0), pv.Bvec(1),
                            pv.Bvec(2), pv.E(0),    pv.E(1),    pv.E(2)};
  for (int i = 0; i < 16; ++i)
    prim[i] = pvals[i];
  rep3[0] = int(rep.status);
  rep3[1] = rep.iters;
  rep3[2] = rep.adjust_cons;
}

ORA_API int ora_c2p_point(int solver, double *cons, const double *g6,
                          const double *seed, const double *atmo, double *prim,
                          int *rep3) {
  return guarded([&] {
    if (axref_params.evolution_eos &&
        CCTK_EQUALS(axref_params.evolution_eos, "Tabulated3d"))
      c2p_point_eos(EOSX::global_eos_3p_tab3d, solver, cons, g6, seed, atmo,
                    prim, rep3);
    else
      c2p_point_eos(EOSX::global_eos_3p_ig, solver, cons, g6, seed, atmo,
                    prim, rep3);
  });
}

// Tabulated EOS queries (EOSX/src/eos_3p_tabulated3d/eos_3p_tabulated3d.hxx:
// 197-340).  which: 0 press(rho,eps,ye) 1 temp(rho,eps,ye) 2 csnd(rho,eps,ye)
// 3 kappa(rho,eps,ye) 4 eps(rho,temp,ye) 5 press(rho,temp,ye)
// 6 entropy(rho,temp,ye).  eps_io is read and, for 0-3, receives the possibly
// clamped eps the reference writes back.
ORA_API double ora_eos_tab_query(int which, double rho, double x, double ye,
                                 double *eps_io) {
  const auto *t = EOSX::global_eos_3p_tab3d;
  double e = x;
  double r = 0;
  switch (which) {
  case 0: r = t->press_from_valid_rho_eps_ye(rho, e, ye); break;
  case 1: r = t->temp_from_valid_rho_eps_ye(rho, e, ye); break;
  case 2: r = t->csnd_from_valid_rho_eps_ye(rho, e, ye); break;
  case 3: r = t->kappa_from_valid_rho_eps_ye(rho, e, ye); break;
  case 4: r = t->eps_from_valid_rho_temp_ye(rho, x, ye); break;
  case 5: r = t->press_from_valid_rho_temp_ye(rho, x, ye); break;
  case 6: r = t->entropy_from_valid_rho_temp_ye(rho, x, ye); break;
  }
  if (eps_io)
    *eps_io = e;
  return r;
}

// ---------------------------------------------------------------------------
// stress-energy tensor and regrid error
// ---------------------------------------------------------------------------
// AsterX_Tmunu (AsterX/src/tmunu.cxx:158-176) at interpolation order 2 or 4.
ORA_API int ora_tmunu(int interp_order) {
  axref_params.tmunu_interp_order = interp_order;
  return guarded([] { AsterX::AsterX_Tmunu(&g_gh); });
}

// The loop of AsterX_EstimateError (AsterX/src/estimate_error.cxx:96-140)
// over the interior cells with the reference's indicators
// (AsterX/src/estimate_error.hxx:14-86), for the grid functions `vars`
// (the box's layout) given directly instead of through the regrid_groups
// parameter; writes regrid_error.
ORA_API int ora_estimate_error(int method, int nvars, double *const *vars,
                               double epsilon_err) {
  return guarded([&] {
    std::vector<Loop::GF3D2<const CCTK_REAL> > gfs;
    for (int i = 0; i < nvars; ++i)
      gfs.emplace_back(vars[i], g_sy, g_sz);
    const Loop::GF3D2<CCTK_REAL> regrid_error(g_fields[AXREF_F_regrid_error], g_sy,
                                              g_sz);
    g_grid.loop_int_device<1, 1, 1>(
        g_grid.nghostzones, [&](const Loop::PointDesc &p) {
          regrid_error(p.I) = 0.0;
          for (int i = 0; i < nvars; i++) {
            CCTK_REAL e = 0;
            switch (method) {
            case AXB_REGRID_FIRST_DERIV: e = AsterX::calc_deriv_1st(gfs[i], p); break;
            case AXB_REGRID_SECOND_DERIV: e = AsterX::calc_deriv_2nd(gfs[i], p); break;
            case AXB_REGRID_SECOND_DERIV_NORM:
              e = AsterX::calc_deriv_2nd_norm(gfs[i], p, epsilon_err);
              break;
            default: e = AsterX::calc_grad_1st(gfs[i], p); break;
            }
            regrid_error(p.I) = std::max({regrid_error(p.I), e});
          }
        });
  });
}
