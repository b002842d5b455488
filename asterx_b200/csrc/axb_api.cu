// C ABI of the engine: contexts, equations of state and the RHS group.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <limits>
#include <new>

#include "axb_batch.cuh"
#include "axb_flux_launch.cuh"
#include "axb_internal.hxx"
#include "axb_rhs_misc.cuh"

using namespace axb;

namespace {

int check_box(const axb_box *b, int min_ng) {
  if (!b)
    return AXB_ERR_ARG;
  for (int d = 0; d < 3; ++d)
    if (b->n[d] < 1 || !(b->dx[d] > 0))
      return AXB_ERR_ARG;
  if (b->ng < min_ng)
    return AXB_ERR_GHOSTS;
  if (b->sy < b->n[0] + 2 * b->ng + 1 || b->sz < b->sy * (b->n[1] + 2 * b->ng + 1))
    return AXB_ERR_ARG;
  return AXB_OK;
}

ReconParams recon_params(const axb_params &p) {
  ReconParams r;
  r.ppm_shock_detection = p.ppm_shock_detection;
  r.ppm_zone_flattening = p.ppm_zone_flattening;
  r.poly_k = p.poly_k;
  r.poly_gamma = p.poly_gamma;
  r.ppm_eta1 = p.ppm_eta1;
  r.ppm_eta2 = p.ppm_eta2;
  r.ppm_eps = p.ppm_eps;
  r.ppm_eps_shock = p.ppm_eps_shock;
  r.ppm_small = p.ppm_small;
  r.ppm_omega1 = p.ppm_omega1;
  r.ppm_omega2 = p.ppm_omega2;
  r.weno_eps = p.weno_eps;
  r.mp5_alpha = p.mp5_alpha;
  return r;
}

#define GFP(name) (f->gf[AXB_GF_##name])

} // namespace

AXB_API void axb_params_default(axb_params *p) {
  std::memset(p, 0, sizeof *p);
  // ReconX/param.ccl
  p->reconstruction_method = AXB_RECON_GODUNOV;
  p->loworder_method = AXB_RECON_GODUNOV;
  p->reconstruct_with_temperature = 0;
  p->ppm_shock_detection = 1;
  p->ppm_zone_flattening = 0;
  p->ppm_eta1 = 20.0;
  p->ppm_eta2 = 0.05;
  p->ppm_eps = 0.33;
  p->ppm_eps_shock = 0.01;
  p->ppm_small = 1e-7;
  p->ppm_omega1 = 0.75;
  p->ppm_omega2 = 10.0;
  p->enhanced_ppm_C2 = 1.25;
  p->weno_eps = 1e-26;
  p->mp5_alpha = 4.0;
  // EOSX/param.ccl
  p->poly_k = 100.0;
  p->poly_gamma = 2.0;
  // AsterX/param.ccl
  p->flux_type = AXB_FLUX_LXF;
  p->recon_type = AXB_RECVAR_V;
  p->vector_potential_gauge = AXB_GAUGE_GEN_LORENZ;
  p->local_spatial_order = 2;
  p->lorenz_damp_fac = 0.0;
  // Con2PrimFactory/param.ccl
  p->c2p_prime = AXB_C2P_NOBLE;
  p->c2p_second = AXB_C2P_PALENZUELA;
  p->max_iter = 30;
  p->thermal_eos_atmo = 1;
  p->c2p_tol = 1e-10;
  p->rho_abs_min = 1e-13;
  p->atmo_tol = 1e-3;
  p->eps_atmo = 1e-10;
  p->p_atmo = 1e-10;
  p->t_atmo = 1e-2;
  p->Ye_atmo = 0.5;
  p->r_atmo = 1e100;
  p->alp_thresh = 0.0;
  p->rho_BH = 1e100;
  p->eps_BH = 1e100;
  p->vwlim_BH = 1e100;
  p->cons_error_limit = -1;
  p->vw_lim = 10.0;
  p->B_lim = 100.0;
}

AXB_API const char *axb_gf_name(int id) {
  static const char *names[] = {
#define AXB_GF_NAME_(name) #name,
      AXB_GF_LIST(AXB_GF_NAME_)
#undef AXB_GF_NAME_
  };
  return (id >= 0 && id < AXB_NUM_GF) ? names[id] : nullptr;
}

namespace axb {
// the context's second stream and its events (created once, on the
// context's device); false when they cannot be had
bool side_stream(axb_ctx *c) {
  if (c->side)
    return true;
  if (!c->allow_side)
    return false;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev != c->device)
    return false;
  if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess) {
    c->side = nullptr;
    return false;
  }
  cudaEvent_t *evs[3] = {&c->ev_fork, &c->ev_sources, &c->ev_aux};
  for (cudaEvent_t *e : evs)
    if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) {
      for (cudaEvent_t *f : evs)
        if (*f)
          cudaEventDestroy(*f);
      c->ev_fork = c->ev_sources = c->ev_aux = nullptr;
      cudaStreamDestroy(c->side);
      c->side = nullptr;
      return false;
    }
  return true;
}

} // namespace axb

AXB_API int axb_ctx_create(int device, axb_ctx **out) {
  if (!out)
    return AXB_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return AXB_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  AXB_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10)
    return AXB_ERR_NO_DEVICE;
  AXB_CUDA_TRY(cudaSetDevice(device));
  axb_ctx *c = new (std::nothrow) axb_ctx();
  if (!c)
    return AXB_ERR_ARG;
  c->device = device;
  if (cudaMalloc(&c->status, sizeof(DevStatus)) != cudaSuccess ||
      cudaMallocHost(&c->status_host_pinned, sizeof(DevStatus)) != cudaSuccess) {
    delete c;
    return AXB_ERR_CUDA;
  }
  AXB_CUDA_TRY(cudaMemset(c->status, 0, sizeof(DevStatus)));
  // the second stream of the RHS group, made here so that no call made
  // during a stream capture has to create it
  c->allow_side = 1;
  if (!side_stream(c))
    c->allow_side = 0;
  *out = c;
  return AXB_OK;
}

AXB_API int axb_ctx_destroy(axb_ctx *c) {
  if (!c)
    return AXB_ERR_ARG;
  if (c->ev) {
    for (int q = 0; q < 2 * AXB_EVENT_POOL; ++q)
      cudaEventDestroy(c->ev[q]);
    delete[] c->ev;
    delete[] c->ev_region;
  }
  if (c->side) {
    cudaStreamSynchronize(c->side);
    cudaStreamDestroy(c->side);
    cudaEventDestroy(c->ev_fork);
    cudaEventDestroy(c->ev_sources);
    cudaEventDestroy(c->ev_aux);
  }
  cudaFree(c->status);
  cudaFreeHost(c->status_host_pinned);
  if (c->pool) {
    cudaDeviceSynchronize(); // stream-ordered frees of the pool's blocks
    cudaMemPoolDestroy(c->pool);
  }
  delete c;
  return AXB_OK;
}

// Start recording a CUDA event pair around every kernel launch of the
// entry points that follow (on their stream).  Creates the event pool on first
// use; call it outside any stream capture.
AXB_API int axb_timing_begin(axb_ctx *c) {
  if (!c)
    return AXB_ERR_ARG;
  if (!c->ev) {
    c->ev = new (std::nothrow) cudaEvent_t[2 * AXB_EVENT_POOL];
    c->ev_region = new (std::nothrow) int[AXB_EVENT_POOL];
    if (!c->ev || !c->ev_region)
      return AXB_ERR_ARG;
    for (int q = 0; q < 2 * AXB_EVENT_POOL; ++q)
      AXB_CUDA_TRY(cudaEventCreate(&c->ev[q]));
  }
  c->ev_used = 0;
  c->timing = 1;
  return AXB_OK;
}

// Stop recording, wait for the recorded launches and return, per kernel
// region (nregions entries: sources, flux x, flux y, flux z, aux, ct+psi,
// rk stage, sync, bstag, c2p, c2p cells, mlp), the summed milliseconds and
// the number of launches.
AXB_API int axb_timing_end(axb_ctx *c, double *ms, int *count, int nregions) {
  if (!c || !ms || !count)
    return AXB_ERR_ARG;
  c->timing = 0;
  for (int r = 0; r < nregions; ++r) {
    ms[r] = 0;
    count[r] = 0;
  }
  if (c->ev_used > 0)
    AXB_CUDA_TRY(cudaEventSynchronize(c->ev[2 * (c->ev_used - 1) + 1]));
  for (int q = 0; q < c->ev_used; ++q) {
    float t = 0;
    AXB_CUDA_TRY(cudaEventElapsedTime(&t, c->ev[2 * q], c->ev[2 * q + 1]));
    const int r = c->ev_region[q];
    if (r < nregions) {
      ms[r] += t;
      count[r] += 1;
    }
  }
  c->ev_used = 0;
  return AXB_OK;
}

// Clear the device error word, CFL maximum and c2p counters (stream-ordered).
AXB_API int axb_status_reset(axb_ctx *c, void *stream) {
  if (!c)
    return AXB_ERR_ARG;
  AXB_CUDA_TRY(cudaMemsetAsync(c->status, 0, sizeof(DevStatus),
                               (cudaStream_t)stream));
  return AXB_OK;
}

// Synchronously read the device status: error word (AXB_EW_* bits), the
// maximum characteristic speed seen by the flux passes since the last reset,
// the number of C2P_FAIL cells, and (optionally, 64 entries) the histogram
// of first-solver iteration counts.
AXB_API int axb_status_read(axb_ctx *c, void *stream, uint32_t *error_word,
                            double *max_speed, uint32_t *c2p_fail,
                            uint64_t *iter_hist64) {
  if (!c)
    return AXB_ERR_ARG;
  AXB_CUDA_TRY(cudaMemcpyAsync(c->status_host_pinned, c->status,
                               sizeof(DevStatus), cudaMemcpyDeviceToHost,
                               (cudaStream_t)stream));
  AXB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  const DevStatus &h = *c->status_host_pinned;
  if (error_word)
    *error_word = h.error_word;
  if (max_speed) {
    const long long bits = (long long)h.max_speed_bits;
    double v;
    std::memcpy(&v, &bits, sizeof v);
    *max_speed = v;
  }
  if (c2p_fail)
    *c2p_fail = h.c2p_fail_count;
  if (iter_hist64)
    for (int i = 0; i < 64; ++i)
      iter_hist64[i] = h.c2p_iter_hist[i];
  return AXB_OK;
}

// Ideal-gas evolution EOS (EOSX_Setup_EOS, EOSX/src/setup_eos.cxx:70-78) plus
// the initial-data polytrope used for a cold atmosphere (:33-41).
AXB_API int axb_eos_create_idealgas(double gamma, double particle_mass,
                                    const double rho_range[2],
                                    const double eps_range[2],
                                    const double ye_range[2], double poly_gamma,
                                    double poly_k, axb_eos **out) {
  if (!out || !rho_range || !eps_range || !ye_range || !(gamma >= 1) ||
      !(poly_gamma > 1))
    return AXB_ERR_ARG;
  axb_eos *e = new (std::nothrow) axb_eos();
  if (!e)
    return AXB_ERR_ARG;
  e->kind = 0;
  e->ideal = make_ideal(gamma, particle_mass, Range{eps_range[0], eps_range[1]},
                        Range{rho_range[0], rho_range[1]},
                        Range{ye_range[0], ye_range[1]});
  e->poly = make_poly(poly_gamma, poly_k);
  e->tab_host = nullptr;
  e->tab_dev = nullptr;
  *out = e;
  return AXB_OK;
}

// Tabulated3d evolution EOS from a table already in memory, in the state
// eos_3p_tabulated3d::init leaves it after reading and converting the file
// (EOSX/src/eos_3p_tabulated3d/eos_3p_tabulated3d.hxx:53-192): natural-log
// axes, 19 variables per node interleaved variable-fastest.  The ranges are
// set up as at the end of init (:179-192), including the eps range of
// compute_eps_range_full_table, which scans the EPS * (node count) block of
// that interleaved array.
namespace {
// Unit factors of EOSX (EOSX/src/utils/eos_constants.hxx:7-14): CGS to the
// code units (G = c = M_sun = 1) the evolution uses.
constexpr double kLengthGF = 6.77269222552442e-06;
constexpr double kTimeGF = 2.03040204956746e05;
constexpr double kRhoGF = 1.61887093132742e-18;
constexpr double kPressGF = 1.80123683248503e-39;
constexpr double kEpsGF = 1.11265005605362e-21;
constexpr int kNTables = 19;
} // namespace

// The conversions eos_3p_tabulated3d::init applies to a StellarCollapse
// table once it has read it
// (EOSX/src/eos_3p_tabulated3d/eos_3p_tabulated3d.hxx:115-177): the 19
// datasets go from one array per variable (rho fastest) to variable-fastest
// nodes, log10 of CGS values become natural logs of code-unit values, cs^2
// and the derivatives get their unit factors, energy_shift becomes code
// units.  Also the ranges init sets (:179-192): rho, temperature, Ye, eps.
AXB_API int axb_eos_stellarcollapse_convert(int nrho, int ntemp, int nye,
                                            const double *logrho10, const double *logtemp10,
                                            const double *ye_in, const double *const *dsets,
                                            double energy_shift_cgs, double *logrho,
                                            double *logtemp, double *ye, double *table,
                                            double *energy_shift, double ranges[8]) {
  if (nrho < 2 || ntemp < 2 || nye < 2 || !logrho10 || !logtemp10 || !ye_in || !dsets ||
      !logrho || !logtemp || !ye || !table || !energy_shift)
    return AXB_ERR_ARG;
  for (int v = 0; v < kNTables; ++v)
    if (!dsets[v])
      return AXB_ERR_ARG;
  const size_t nodes = size_t(nrho) * ntemp * nye;
  const double ln10 = std::log(10.0);
  const double inv_time2 = 1 / (kTimeGF * kTimeGF);
  *energy_shift = energy_shift_cgs * kEpsGF;
  const double lrho = std::log(kRhoGF);
  for (int q = 0; q < nrho; ++q)
    logrho[q] = logrho10[q] * ln10 + lrho;
  for (int q = 0; q < ntemp; ++q)
    logtemp[q] = logtemp10[q] * ln10;
  for (int q = 0; q < nye; ++q)
    ye[q] = ye_in[q];
  const double lpress = std::log(kPressGF), leps = std::log(kEpsGF);
  for (size_t n = 0; n < nodes; ++n) {
    double *t = table + kNTables * n;
    for (int v = 0; v < kNTables; ++v)
      t[v] = dsets[v][n];
    t[0] = t[0] * ln10 + lpress;                              // ln press
    t[1] = t[1] * ln10 + leps;                                // ln(eps + shift)
    t[4] = t[4] * kLengthGF * kLengthGF * inv_time2;           // cs^2
    t[5] = t[5] * kEpsGF;                                     // d eps / dT
    t[6] = t[6] * kPressGF / kRhoGF;                          // dp/drho at eps
    t[7] = t[7] * kPressGF / kEpsGF;                          // dp/deps at rho
  }
  if (ranges) {
    ranges[0] = std::exp(logrho[0]);
    ranges[1] = std::exp(logrho[nrho - 1]);
    ranges[2] = std::exp(logtemp[0]);
    ranges[3] = std::exp(logtemp[ntemp - 1]);
    ranges[4] = ye[0];
    ranges[5] = ye[nye - 1];
    // compute_eps_range_full_table (eos_3p_tabulated3d.hxx:447-458): the
    // extremes of exp(ln(eps + shift)) - shift over the table's nodes, with
    // the table read in its variable-major order as the reference reads it
    double emin = std::numeric_limits<double>::max();
    double emax = std::numeric_limits<double>::lowest();
    for (size_t n = 0; n < nodes; ++n) {
      const double e = std::exp(table[1 * nodes + n]) - *energy_shift;
      emin = std::fmin(emin, e);
      emax = std::fmax(emax, e);
    }
    ranges[6] = std::fmax(emin, 1e-15);
    ranges[7] = emax;
  }
  return AXB_OK;
}

AXB_API int axb_eos_create_tabulated3d(int nrho, int ntemp, int nye,
                                       const double *logrho, const double *logtemp,
                                       const double *ye, const double *table,
                                       double energy_shift, double poly_gamma,
                                       double poly_k, axb_eos **out) {
  if (!out || !logrho || !logtemp || !ye || !table || nrho < 2 || ntemp < 2 ||
      nye < 2 || !(poly_gamma > 1))
    return AXB_ERR_ARG;
  const int nax[3] = {nrho, ntemp, nye};
  const double *ax[3] = {logrho, logtemp, ye};
  for (int d = 0; d < 3; ++d)
    if (!(ax[d][1] > ax[d][0]))
      return AXB_ERR_ARG;
  const size_t nodes = size_t(nrho) * ntemp * nye;
  // the table starts on a 32-byte sector: axes padded to 4 doubles
  const size_t naxes = (size_t(nrho) + ntemp + nye + 3) / 4 * 4;
  const size_t total = naxes + nodes * TAB_NV;
  double *h = static_cast<double *>(std::malloc(total * sizeof(double)));
  if (!h)
    return AXB_ERR_ARG;
  double *dptr = nullptr;
  if (cudaMalloc(&dptr, total * sizeof(double)) != cudaSuccess) {
    std::free(h);
    return AXB_ERR_CUDA;
  }
  size_t o = 0;
  double *hx[3];
  for (int d = 0; d < 3; ++d) {
    hx[d] = h + o;
    std::memcpy(hx[d], ax[d], nax[d] * sizeof(double));
    o += nax[d];
  }
  double *hy = h + naxes;
  const int keep[TAB_NV] = {0, 1, 2, 4}; // ln P, ln(eps + shift), s, cs^2
  for (size_t q = 0; q < nodes; ++q)
    for (int v = 0; v < TAB_NV; ++v)
      hy[TAB_NV * q + v] = table[size_t(19) * q + keep[v]];
  EosTab t{};
  for (int d = 0; d < 3; ++d) {
    t.n[d] = nax[d];
    t.x[d] = hx[d];
    t.idx[d] = 1. / (ax[d][1] - ax[d][0]);
    t.x0[d] = ax[d][0];
    t.xlast[d] = ax[d][nax[d] - 1];
  }
  t.y = hy;
  t.shift = energy_shift;
  t.rgrho = Range{std::exp(t.x0[0]), std::exp(t.xlast[0])};
  t.rgtemp = Range{std::exp(t.x0[1]), std::exp(t.xlast[1])};
  t.rgye = Range{t.x0[2], t.xlast[2]};
  double emin = std::numeric_limits<double>::max();
  double emax = std::numeric_limits<double>::lowest();
  for (size_t q = 0; q < nodes; ++q) {
    const double v = std::exp(table[1 * nodes + q]) - energy_shift;
    emin = std::fmin(emin, v);
    emax = std::fmax(emax, v);
  }
  t.rgeps = Range{std::fmax(emin, 1e-15), emax};
  t.err = nullptr;
  if (cudaMemcpy(dptr, h, total * sizeof(double), cudaMemcpyHostToDevice) !=
      cudaSuccess) {
    cudaFree(dptr);
    std::free(h);
    return AXB_ERR_CUDA;
  }
  axb_eos *e = new (std::nothrow) axb_eos();
  if (!e) {
    cudaFree(dptr);
    std::free(h);
    return AXB_ERR_ARG;
  }
  e->kind = 1;
  e->ideal = EosIdeal{};
  e->poly = make_poly(poly_gamma, poly_k);
  e->tab_h = t;
  e->tab_d = t;
  for (int d = 0; d < 3; ++d)
    e->tab_d.x[d] = dptr + (hx[d] - h);
  e->tab_d.y = dptr + (hy - h);
  e->tab_host = h;
  e->tab_dev = dptr;
  *out = e;
  return AXB_OK;
}

// A StellarCollapse table as its file holds it (the datasets' values, see
// axb_eos_stellarcollapse_convert) to the device EOS: the conversion of
// eos_3p_tabulated3d::init, then axb_eos_create_tabulated3d.
AXB_API int axb_eos_create_stellarcollapse(int nrho, int ntemp, int nye,
                                           const double *logrho10, const double *logtemp10,
                                           const double *ye_in, const double *const *dsets,
                                           double energy_shift_cgs, double poly_gamma,
                                           double poly_k, axb_eos **out) {
  if (!out || nrho < 2 || ntemp < 2 || nye < 2)
    return AXB_ERR_ARG;
  const size_t nodes = size_t(nrho) * ntemp * nye;
  std::vector<double> lr(nrho), lt(ntemp), y(nye);
  std::vector<double> table;
  try {
    table.resize(nodes * kNTables);
  } catch (const std::bad_alloc &) {
    return AXB_ERR_TOO_LARGE;
  }
  double shift = 0.0;
  int rc = axb_eos_stellarcollapse_convert(nrho, ntemp, nye, logrho10, logtemp10, ye_in, dsets,
                                           energy_shift_cgs, lr.data(), lt.data(), y.data(),
                                           table.data(), &shift, nullptr);
  if (rc)
    return rc;
  return axb_eos_create_tabulated3d(nrho, ntemp, nye, lr.data(), lt.data(), y.data(),
                                    table.data(), shift, poly_gamma, poly_k, out);
}

AXB_API int axb_eos_destroy(axb_eos *e) {
  if (!e)
    return AXB_ERR_ARG;
  if (e->tab_dev)
    cudaFree(e->tab_dev);
  std::free(e->tab_host);
  delete e;
  return AXB_OK;
}

namespace {
int fill_rhs_args(axb_ctx *c, const axb_box *box, const axb_fields *f,
                  const axb_params *p, RhsArgs &a) {
  int rc = check_box(box, 3);
  if (rc)
    return rc;
  if (!f || !p)
    return AXB_ERR_ARG;
  if (p->recon_type < AXB_RECVAR_V || p->recon_type > AXB_RECVAR_S ||
      p->reconstruction_method == AXB_RECON_EPPM ||
      !(p->local_spatial_order == 2 || p->local_spatial_order == 4))
    return AXB_ERR_UNSUPPORTED;
  if (p->local_spatial_order == 4 && box->ng < 3)
    return AXB_ERR_GHOSTS;
  a.b = make_box(*box);
  // no fused stage unless the caller sets one up (axb_substep)
  a.fuse_stage = 0;
  a.st_alpha = a.st_beta = a.st_gdt = 0.0;
  for (int v = 0; v < 11; ++v) {
    a.st_un[v] = nullptr;
    a.st_uk[v] = nullptr;
  }
  a.rho = GFP(rho);
  a.vel[0] = GFP(velx);
  a.vel[1] = GFP(vely);
  a.vel[2] = GFP(velz);
  a.recvar = p->recon_type;
  for (int q = 0; q < 3; ++q)
    a.recv[q] = p->recon_type == AXB_RECVAR_Z   ? f->gf[AXB_GF_zvec_x + q]
                : p->recon_type == AXB_RECVAR_S ? f->gf[AXB_GF_svec_x + q]
                                                : a.vel[q];
  a.eps = GFP(eps);
  a.press = GFP(press);
  a.temperature = GFP(temperature);
  a.rec_temp = p->reconstruct_with_temperature != 0;
  a.thermo = a.rec_temp ? a.temperature : a.press;
  a.Ye = GFP(Ye);
  a.entropy = GFP(entropy);
  a.Bvec[0] = GFP(Bvecx);
  a.Bvec[1] = GFP(Bvecy);
  a.Bvec[2] = GFP(Bvecz);
  a.dBstag[0] = GFP(dBx_stag);
  a.dBstag[1] = GFP(dBy_stag);
  a.dBstag[2] = GFP(dBz_stag);
  a.alp = GFP(alp);
  a.beta[0] = GFP(betax);
  a.beta[1] = GFP(betay);
  a.beta[2] = GFP(betaz);
  const int gid[6] = {AXB_GF_gxx, AXB_GF_gxy, AXB_GF_gxz, AXB_GF_gyy, AXB_GF_gyz, AXB_GF_gzz};
  const int kid[6] = {AXB_GF_kxx, AXB_GF_kxy, AXB_GF_kxz, AXB_GF_kyy, AXB_GF_kyz, AXB_GF_kzz};
  for (int q = 0; q < 6; ++q) {
    a.g[q] = f->gf[gid[q]];
    a.K[q] = f->gf[kid[q]];
  }
  a.Avec[0] = GFP(Avec_x);
  a.Avec[1] = GFP(Avec_y);
  a.Avec[2] = GFP(Avec_z);
  a.Psi = GFP(Psi);
  const int accid[7] = {AXB_GF_acc_dens, AXB_GF_acc_momx, AXB_GF_acc_momy,
                        AXB_GF_acc_momz, AXB_GF_acc_tau,  AXB_GF_acc_DYe,
                        AXB_GF_acc_DEnt};
  const int rhsid[7] = {AXB_GF_densrhs, AXB_GF_momxrhs, AXB_GF_momyrhs,
                        AXB_GF_momzrhs, AXB_GF_taurhs,  AXB_GF_DYe_rhs,
                        AXB_GF_DEntrhs};
  for (int q = 0; q < 7; ++q) {
    a.acc[q] = f->gf[accid[q]];
    a.rhs[q] = f->gf[rhsid[q]];
  }
  const int bfid[6] = {AXB_GF_fxBy, AXB_GF_fxBz, AXB_GF_fyBx,
                       AXB_GF_fyBz, AXB_GF_fzBx, AXB_GF_fzBy};
  for (int q = 0; q < 6; ++q)
    a.bflux[q] = f->gf[bfid[q]];
  const int auxid[7] = {AXB_GF_Fx, AXB_GF_Fy, AXB_GF_Fz, AXB_GF_Fbetax,
                        AXB_GF_Fbetay, AXB_GF_Fbetaz, AXB_GF_G};
  for (int q = 0; q < 7; ++q)
    a.aux[q] = f->gf[auxid[q]];
  // upwind CT: per face direction vtilde^{d+1}, vtilde^{d+2}, amax, amin
  static const int uctid[12] = {
      AXB_GF_vtilde_y_xface, AXB_GF_vtilde_z_xface, AXB_GF_amax_xface, AXB_GF_amin_xface,
      AXB_GF_vtilde_z_yface, AXB_GF_vtilde_x_yface, AXB_GF_amax_yface, AXB_GF_amin_yface,
      AXB_GF_vtilde_x_zface, AXB_GF_vtilde_y_zface, AXB_GF_amax_zface, AXB_GF_amin_zface};
  a.use_uct = p->use_uct != 0;
  for (int q = 0; q < 12; ++q)
    a.uct[q] = a.use_uct ? f->gf[uctid[q]] : nullptr;
  // the flux passes cover 1 transverse ghost layer, 3 with upwind CT
  a.text = a.use_uct ? 3 : 1;
  a.recon_method = p->reconstruction_method;
  a.Arhs[0] = GFP(Avec_x_rhs);
  a.Arhs[1] = GFP(Avec_y_rhs);
  a.Arhs[2] = GFP(Avec_z_rhs);
  a.Psi_rhs = GFP(Psi_rhs);
  a.rp = recon_params(*p);
  a.recon_lo = p->loworder_method;
  a.flux_type = p->flux_type;
  a.gauge = p->vector_potential_gauge;
  a.fd_order = p->local_spatial_order;
  a.lorenz_damp_fac = p->lorenz_damp_fac;
  a.write_bflux = 1;
  a.status = c->status;
  // every pointer the group reads or writes must be present
  const void *req[] = {a.rho, a.vel[0], a.vel[1], a.vel[2], a.eps, a.press, a.thermo,
                       a.Ye, a.entropy, a.Bvec[0], a.Bvec[1], a.Bvec[2],
                       a.dBstag[0], a.dBstag[1], a.dBstag[2], a.alp, a.beta[0],
                       a.beta[1], a.beta[2], a.Avec[0], a.Avec[1], a.Avec[2],
                       a.Psi, a.Arhs[0], a.Arhs[1], a.Arhs[2], a.Psi_rhs};
  for (const void *q : req)
    if (!q)
      return AXB_ERR_ARG;
  for (int q = 0; q < 6; ++q)
    if (!a.g[q] || !a.K[q] || !a.bflux[q])
      return AXB_ERR_ARG;
  for (int q = 0; q < 7; ++q)
    if (!a.acc[q] || !a.rhs[q] || !a.aux[q])
      return AXB_ERR_ARG;
  for (int q = 0; q < 3; ++q)
    if (!a.recv[q])
      return AXB_ERR_ARG;
  for (int q = 0; q < 12; ++q)
    if (a.use_uct && !a.uct[q])
      return AXB_ERR_ARG;
  return AXB_OK;
}
} // namespace

namespace axb {
int launch_flux_pass(int dir, int recon, const RhsArgs &a, const axb_eos &eos,
                     int seglen, cudaStream_t s) {
  switch (recon) {
  case AXB_RECON_PPM: return launch_flux_ppm(dir, a, eos, seglen, s);
  case AXB_RECON_WENOZ: return launch_flux_wenoz(dir, a, eos, seglen, s);
  case AXB_RECON_MP5: return launch_flux_mp5(dir, a, eos, seglen, s);
  default: return launch_flux_low(recon, dir, a, eos, seglen, s);
  }
}
} // namespace axb

namespace {
// The stage update a substep fuses into its RHS group.
struct StageFuse {
  const axb_fields *un;
  double alpha, beta, gdt;
};

int rhs_group_run(axb_ctx *c, const axb_box *box, const axb_fields *f,
                  const axb_params *p, const axb_eos *eos, void *stream,
                  const StageFuse *fuse, const int *bc = nullptr) {
  if (!c || !eos)
    return AXB_ERR_ARG;
  RhsArgs a;
  int rc = fill_rhs_args(c, box, f, p, a);
  if (rc)
    return rc;
  a.fuse_stage = 0;
  if (fuse) {
    static const int evolved[11] = {AXB_GF_dens,   AXB_GF_momx,   AXB_GF_momy,
                                    AXB_GF_momz,   AXB_GF_tau,    AXB_GF_DYe,
                                    AXB_GF_DEnt,   AXB_GF_Avec_x, AXB_GF_Avec_y,
                                    AXB_GF_Avec_z, AXB_GF_Psi};
    if (!fuse->un)
      return AXB_ERR_ARG;
    for (int v = 0; v < 11; ++v) {
      a.st_un[v] = fuse->un->gf[evolved[v]];
      a.st_uk[v] = f->gf[evolved[v]];
      if (!a.st_un[v] || !a.st_uk[v])
        return AXB_ERR_ARG;
    }
    a.fuse_stage = 1;
    a.st_alpha = fuse->alpha;
    a.st_beta = fuse->beta;
    a.st_gdt = fuse->gdt;
  }
  // the tabulated EOS has no eps(rho, press) (the reference asserts,
  // eos_3p_tabulated3d.hxx:259-269): its fluxes need the reconstructed
  // temperature
  if (eos->kind == 1 && !a.rec_temp)
    return AXB_ERR_UNSUPPORTED;
  cudaStream_t s = (cudaStream_t)stream;
#ifndef AXB_FLUX_SEGLEN
#define AXB_FLUX_SEGLEN 16 // cells per y/z pencil segment (one thread each)
#endif
  const int seglen = AXB_FLUX_SEGLEN;
  if (!bc && side_stream(c)) {
    // the sources and the vertex auxiliaries read neither the partial
    // divergences nor the face B fluxes, and the flux passes read neither
    // the sources' RHS nor the auxiliaries: they run on the second stream
    // beside the x and y passes; the z pass waits for the sources' RHS, the
    // CT kernel for the auxiliaries (which read A and Psi before it
    // updates them)
    cudaEventRecord(c->ev_fork, s);
    cudaStreamWaitEvent(c->side, c->ev_fork, 0);
    axb_mark(c, AXB_R_SOURCES, c->side, true);
    rc = launch_rhs_misc(p->local_spatial_order == 4 ? 1 : 0, a, c->side);
    axb_mark(c, AXB_R_SOURCES, c->side, false);
    cudaEventRecord(c->ev_sources, c->side);
    int rc_aux = AXB_OK;
    if (!rc) {
      axb_mark(c, AXB_R_AUX, c->side, true);
      rc_aux = launch_rhs_misc(2, a, c->side);
      axb_mark(c, AXB_R_AUX, c->side, false);
    }
    cudaEventRecord(c->ev_aux, c->side);
    for (int dir = 0; dir < 3 && !rc && !rc_aux; ++dir) {
      if (dir == 2)
        cudaStreamWaitEvent(s, c->ev_sources, 0);
      axb_mark(c, AXB_R_FLUX_X + dir, s, true);
      rc = launch_flux_pass(dir, p->reconstruction_method, a, *eos, seglen, s);
      axb_mark(c, AXB_R_FLUX_X + dir, s, false);
    }
    // always joined back, on success or not
    cudaStreamWaitEvent(s, c->ev_aux, 0);
    if (rc || rc_aux)
      return rc ? rc : rc_aux;
    axb_mark(c, AXB_R_CT, s, true);
    rc = launch_rhs_misc(3, a, s);
    axb_mark(c, AXB_R_CT, s, false);
    return rc;
  }
  axb_mark(c, AXB_R_SOURCES, s, true);
  rc = launch_rhs_misc(p->local_spatial_order == 4 ? 1 : 0, a, s);
  axb_mark(c, AXB_R_SOURCES, s, false);
  if (rc)
    return rc;
  for (int dir = 0; dir < 3; ++dir) {
    axb_mark(c, AXB_R_FLUX_X + dir, s, true);
    rc = launch_flux_pass(dir, p->reconstruction_method, a, *eos, seglen, s);
    axb_mark(c, AXB_R_FLUX_X + dir, s, false);
    if (rc)
      return rc;
  }
  // physical outer boundaries: the face B fluxes of the ghost layers by the
  // boundary rule, as the reference SYNCs its face fluxes
  static const int bflux_ids[6] = {AXB_GF_fxBy, AXB_GF_fxBz, AXB_GF_fyBx,
                                   AXB_GF_fyBz, AXB_GF_fzBx, AXB_GF_fzBy};
  static const int aux_ids[7] = {AXB_GF_Fx, AXB_GF_Fy, AXB_GF_Fz, AXB_GF_Fbetax,
                                 AXB_GF_Fbetay, AXB_GF_Fbetaz, AXB_GF_G};
  if (bc && (rc = axb_fill_boundary(c, box, f, bflux_ids, 6, bc, stream)))
    return rc;
  // upwind CT: its face data of the ghost layers likewise (the reference
  // SYNCs vtilde_*face and a_*face, AsterX/schedule.ccl:189-193)
  static const int uct_ids[12] = {
      AXB_GF_vtilde_y_xface, AXB_GF_vtilde_z_xface, AXB_GF_amax_xface, AXB_GF_amin_xface,
      AXB_GF_vtilde_z_yface, AXB_GF_vtilde_x_yface, AXB_GF_amax_yface, AXB_GF_amin_yface,
      AXB_GF_vtilde_x_zface, AXB_GF_vtilde_y_zface, AXB_GF_amax_zface, AXB_GF_amin_zface};
  if (bc && a.use_uct && (rc = axb_fill_boundary(c, box, f, uct_ids, 12, bc, stream)))
    return rc;
  axb_mark(c, AXB_R_AUX, s, true);
  rc = launch_rhs_misc(2, a, s);
  axb_mark(c, AXB_R_AUX, s, false);
  if (rc)
    return rc;
  if (bc && (rc = axb_fill_boundary(c, box, f, aux_ids, 7, bc, stream)))
    return rc;
  axb_mark(c, AXB_R_CT, s, true);
  rc = launch_rhs_misc(3, a, s);
  axb_mark(c, AXB_R_CT, s, false);
  return rc;
}
} // namespace

// AsterX_RHSGroup (AsterX/schedule.ccl:169-228): AsterX_Fluxes
// (fluxes.cxx:828-878), AsterX_SourceTerms (source.cxx:170-185) and
// AsterX_RHS (rhs.cxx:18-253) on one box.  Writes densrhs..DEntrhs,
// Avec_*_rhs and Psi_rhs on the interior; uses the scratch grid functions
// acc_*, fxBy..fzBy and Fx..G.  Asynchronous on `stream`.
AXB_API int axb_rhs_group(axb_ctx *c, const axb_box *box, const axb_fields *f,
                          const axb_params *p, const axb_eos *eos, void *stream) {
  return rhs_group_run(c, box, f, p, eos, stream, nullptr);
}

// AsterX_RHSGroup on a box with physical outer boundaries: the face B
// fluxes and the vertex auxiliaries of the ghost points come from the
// boundary rule applied to their interior values (the reference computes
// them on the interior and SYNCs them, AsterX/schedule.ccl:174-195).
AXB_API int axb_rhs_group_bc(axb_ctx *c, const axb_box *box, const axb_fields *f,
                             const axb_params *p, const axb_eos *eos, const int bc[6],
                             void *stream) {
  if (!bc)
    return AXB_ERR_ARG;
  return rhs_group_run(c, box, f, p, eos, stream, nullptr, bc);
}

namespace axb {
// 0: sources FD2, 1: sources FD4, 2: aux, 3: CT + Psi
int launch_rhs_misc(int which, const RhsArgs &a, cudaStream_t s) {
  const BoxDev &b = a.b;
  const int T = 128;
  if (which <= 1 && AXB_SOURCES_SEG > 1) {
    const int seg = AXB_SOURCES_SEG;
    const dim3 grid((b.n[0] + T - 1) / T, b.n[1], (b.n[2] + seg - 1) / seg);
    if (which == 0)
      k_sources_column<2><<<grid, T, 0, s>>>(a, seg);
    else
      k_sources_column<4><<<grid, T, 0, s>>>(a, seg);
  } else if (which <= 1) {
    const dim3 grid((b.n[0] + T - 1) / T, b.n[1], b.n[2]);
    if (which == 0)
      k_sources<2><<<grid, T, 0, s>>>(a);
    else
      k_sources<4><<<grid, T, 0, s>>>(a);
  } else {
    // vertex and edge kernels: threads walk the (i, j) plane row after row,
    // so rows of n+5 or n+1 points do not leave a block mostly idle
    RhsArgs ap = a;
    ap.b.packed = 1;
    const int e = which == 2 ? 5 : 1;
    const long long plane = (long long)(b.n[0] + e) * (b.n[1] + e);
    const dim3 grid(unsigned((plane + T - 1) / T), 1, b.n[2] + e);
    if (which == 2)
      k_aux<<<grid, T, 0, s>>>(ap);
    else if (!a.use_uct)
      k_ct_psi<<<grid, T, 0, s>>>(ap);
    else {
      switch (a.recon_method) {
      case AXB_RECON_GODUNOV: k_ct_psi_uct<AXB_RECON_GODUNOV><<<grid, T, 0, s>>>(ap); break;
      case AXB_RECON_MINMOD: k_ct_psi_uct<AXB_RECON_MINMOD><<<grid, T, 0, s>>>(ap); break;
      case AXB_RECON_MONOCENTRAL:
        k_ct_psi_uct<AXB_RECON_MONOCENTRAL><<<grid, T, 0, s>>>(ap);
        break;
      case AXB_RECON_PPM: k_ct_psi_uct<AXB_RECON_PPM><<<grid, T, 0, s>>>(ap); break;
      case AXB_RECON_WENOZ: k_ct_psi_uct<AXB_RECON_WENOZ><<<grid, T, 0, s>>>(ap); break;
      case AXB_RECON_MP5: k_ct_psi_uct<AXB_RECON_MP5><<<grid, T, 0, s>>>(ap); break;
      default: return AXB_ERR_UNSUPPORTED;
      }
    }
  }
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}
} // namespace axb

// ---------------------------------------------------------------------------
// batched forms (see axb_batch.cuh)
// ---------------------------------------------------------------------------
namespace {
template <int FD>
__global__ void __launch_bounds__(128, AXB_SOURCES_MINB)
    k_sources_batch(const RhsArgs *args, const TileTable t, unsigned long long *ctr) {
  batch_loop(args, t, ctr, [&](const RhsArgs &a, const uint3 bid) {
    if (AXB_SOURCES_SEG > 1)
      sources_column<FD>(a, bid, AXB_SOURCES_SEG);
    else
      sources_body<FD>(a, bid);
  });
}
__global__ void __launch_bounds__(128) k_aux_batch(const RhsArgs *args, const TileTable t, unsigned long long *ctr) {
  batch_loop(args, t, ctr, [&](const RhsArgs &a, const uint3 bid) { aux_body(a, bid); });
}
__global__ void __launch_bounds__(128) k_ct_psi_batch(const RhsArgs *args, const TileTable t, unsigned long long *ctr) {
  batch_loop(args, t, ctr, [&](const RhsArgs &a, const uint3 bid) { ct_psi_body<-1>(a, bid); });
}
} // namespace

namespace axb {
// The per-box RHS argument blocks of a batch (checked as axb_rhs_group
// checks them), in device memory.
int batch_rhs_setup(axb_ctx *c, int nbox, const axb_box *boxes, const axb_fields *f,
                    const axb_params *p, const axb_eos *eos, void **out) {
  *out = nullptr;
  RhsArgs *h = new (std::nothrow) RhsArgs[nbox];
  if (!h)
    return AXB_ERR_ARG;
  for (int b = 0; b < nbox; ++b) {
    int rc = fill_rhs_args(c, boxes + b, f + b, p, h[b]);
    if (!rc && p->use_uct)
      rc = AXB_ERR_UNSUPPORTED; // the batched CT kernel is flux CT only
    h[b].b.packed = 1;
    if (!rc && eos->kind == 1 && !h[b].rec_temp)
      rc = AXB_ERR_UNSUPPORTED;
    if (rc) {
      delete[] h;
      return rc;
    }
  }
  int rc = AXB_OK;
  if (cudaMalloc(out, nbox * sizeof(RhsArgs)) != cudaSuccess ||
      cudaMemcpy(*out, h, nbox * sizeof(RhsArgs), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = AXB_ERR_CUDA;
  delete[] h;
  return rc;
}

// batched grids over packed (i, j) planes: 0 sources, 2 aux, 3 CT + Psi
uint3 rhs_misc_grid(int which, const axb_box &b) {
  const int T = 128;
  const int e = which <= 1 ? 0 : which == 2 ? 5 : 1;
  const long long plane = (long long)(b.n[0] + e) * (b.n[1] + e);
  if (which <= 1 && AXB_SOURCES_SEG > 1) // z columns of the sources
    return make_uint3(unsigned((plane + T - 1) / T), 1,
                      (b.n[2] + AXB_SOURCES_SEG - 1) / AXB_SOURCES_SEG);
  return make_uint3(unsigned((plane + T - 1) / T), 1, b.n[2] + e);
}

int launch_rhs_misc_batch(int which, const void *args, const TileTable &t,
                          unsigned long long *ctr, int nblocks, cudaStream_t s) {
  if (t.total == 0)
    return AXB_OK;
  const RhsArgs *a = static_cast<const RhsArgs *>(args);
  if (which == 0)
    k_sources_batch<2><<<nblocks, 128, 0, s>>>(a, t, ctr);
  else if (which == 1)
    k_sources_batch<4><<<nblocks, 128, 0, s>>>(a, t, ctr);
  else if (which == 2)
    k_aux_batch<<<nblocks, 128, 0, s>>>(a, t, ctr);
  else
    k_ct_psi_batch<<<nblocks, 128, 0, s>>>(a, t, ctr);
  return cudaGetLastError() == cudaSuccess ? AXB_OK : AXB_ERR_CUDA;
}

using Ctr = unsigned long long;
int launch_flux_batch_ppm(int, const RhsArgs *, const TileTable &, Ctr *, const axb_eos &,
                          DevStatus *, int, int, cudaStream_t);
int launch_flux_batch_wenoz(int, const RhsArgs *, const TileTable &, Ctr *, const axb_eos &,
                            DevStatus *, int, int, cudaStream_t);
int launch_flux_batch_mp5(int, const RhsArgs *, const TileTable &, Ctr *, const axb_eos &,
                          DevStatus *, int, int, cudaStream_t);
int launch_flux_batch_low(int, int, const RhsArgs *, const TileTable &, Ctr *,
                          const axb_eos &, DevStatus *, int, int, cudaStream_t);

int launch_flux_batch(int recon, int dir, const RhsArgs *args, const TileTable &t, Ctr *ctr,
                      const axb_eos &eos, DevStatus *st, int seglen, int nblocks,
                      cudaStream_t s) {
  switch (recon) {
  case AXB_RECON_PPM:
    return launch_flux_batch_ppm(dir, args, t, ctr, eos, st, seglen, nblocks, s);
  case AXB_RECON_WENOZ:
    return launch_flux_batch_wenoz(dir, args, t, ctr, eos, st, seglen, nblocks, s);
  case AXB_RECON_MP5:
    return launch_flux_batch_mp5(dir, args, t, ctr, eos, st, seglen, nblocks, s);
  default:
    return launch_flux_batch_low(recon, dir, args, t, ctr, eos, st, seglen, nblocks, s);
  }
}

// batched grid of a flux pass: the x pass as launch_flux_pass_eos (a 1-D
// grid of 4-warp blocks over the rows), the y and z passes over the packed
// transverse plane (128 pencils per block) times the segments along dir
uint3 flux_grid(int dir, const axb_box &b, int seglen) {
  if (dir == 0) {
    const long long warps = (long long)(b.n[1] + 2) * (b.n[2] + 2);
    return make_uint3(unsigned((warps * 32 + 127) / 128), 1, 1);
  }
  const int T1 = dir == 2 ? 1 : 2;
  const long long plane = (long long)(b.n[0] + 2) * (b.n[T1] + 2);
  return make_uint3(unsigned((plane + 127) / 128), 1, (b.n[dir] + seglen - 1) / seglen);
}
} // namespace axb

extern "C" int axb_con2prim_group(axb_ctx *, const axb_box *, const axb_fields *,
                                  const axb_params *, const axb_eos *, void *);
extern "C" int axb_rk_stage(axb_ctx *, const axb_box *, const axb_fields *,
                            const axb_fields *, const axb_fields *,
                            const axb_fields *, double, double, double, double,
                            void *);
extern "C" int axb_sync_periodic(axb_ctx *, const axb_box *, const axb_fields *,
                                 const int *, int, void *);

// One Runge-Kutta substep of one box: the RHS group and the stage update
//   U_k <- alpha U_n + beta U_k + gamma dt RHS(U_k)
// (fused: the RHS grid functions are not written),
// a periodic ghost fill of the evolved variables (when `periodic`), the
// post-step group (curl A, dB, con2prim) and a periodic ghost fill of the
// primitives.  `f` holds U_k (updated in place), the primitives and the
// scratch; `fn` holds U_n (only its 11 evolved grid functions are read).
// Graph-capturable: no allocation and no host synchronisation.
AXB_API int axb_substep(axb_ctx *c, const axb_box *box, const axb_fields *f,
                        const axb_fields *fn, const axb_params *p,
                        const axb_eos *eos, double alpha, double beta,
                        double gamma, double dt, int periodic, void *stream) {
  // the RHS group with the stage update fused into its last kernels: the
  // z flux pass updates the hydro variables, the CT kernel A and Psi, and
  // no RHS grid function is stored (the same bits as axb_rhs_group followed
  // by axb_rk_stage)
  const StageFuse fuse{fn, alpha, beta, gamma * dt};
  int rc = rhs_group_run(c, box, f, p, eos, stream, &fuse);
  if (rc)
    return rc;
  if (periodic) {
    static const int evolved[] = {AXB_GF_dens,   AXB_GF_momx,   AXB_GF_momy,
                                  AXB_GF_momz,   AXB_GF_tau,    AXB_GF_DYe,
                                  AXB_GF_DEnt,   AXB_GF_Avec_x, AXB_GF_Avec_y,
                                  AXB_GF_Avec_z, AXB_GF_Psi};
    if ((rc = axb_sync_periodic(c, box, f, evolved, 11, stream)))
      return rc;
  }
  if ((rc = axb_con2prim_group(c, box, f, p, eos, stream)))
    return rc;
  if (periodic) {
    // the primitives, and the zvec or svec the fluxes reconstruct instead
    // of the velocity when recon_type asks for one of them
    int prims[15] = {AXB_GF_rho,   AXB_GF_velx,    AXB_GF_vely,
                     AXB_GF_velz,  AXB_GF_eps,     AXB_GF_press,
                     AXB_GF_temperature, AXB_GF_Ye, AXB_GF_entropy,
                     AXB_GF_Bvecx, AXB_GF_Bvecy,   AXB_GF_Bvecz};
    int nprims = 12;
    if (p->recon_type == AXB_RECVAR_Z || p->recon_type == AXB_RECVAR_S) {
      const int first = p->recon_type == AXB_RECVAR_Z ? AXB_GF_zvec_x : AXB_GF_svec_x;
      for (int q = 0; q < 3; ++q)
        prims[nprims++] = first + q;
    }
    if ((rc = axb_sync_periodic(c, box, f, prims, nprims, stream)))
      return rc;
  }
  return AXB_OK;
}
