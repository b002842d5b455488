/*
 * asterx_b200.h -- C ABI of the B200 (sm_100a) GRMHD right-hand-side and
 * primitive-recovery engine.
 *
 * The engine is a drop-in for the scheduled hot path of AsterX (Valencia
 * GRMHD with a staggered vector potential): the ReconX reconstruction, the
 * AsterX flux / source / RHS routines with flux-CT and generalised Lorenz
 * gauge, the curl(A) -> B post-step and the Con2PrimFactory Noble and
 * Palenzuela recoveries with the EOSX ideal-gas and tabulated3d equations of
 * state.  Every entry point takes plain pointers and sizes, runs
 * asynchronously on the caller's CUDA stream, allocates nothing on the hot
 * path and returns an int status (0 = success, see axb_status).  All
 * arithmetic is FP64; only the learned c2p guess runs in BF16/FP32.
 *
 * Data model (the CarpetX conventions the reference code assumes):
 *  - A box has n[d] interior cells and ng ghost layers per axis.  Every grid
 *    function of the box is one FP64 array addressed as
 *        f[i + sy*j + sz*k],  0 <= i,j,k <= n[d] + 2*ng,
 *    whatever its centring.  Cell i lies between vertices i and i+1; face i
 *    along an axis is the lower face of cell i; an x-edge (i,j,k) is
 *    cell-centred in x and vertex-centred in y and z (AsterX/interface.ccl:
 *    39-83,102).  Interior cells are [ng, ng+n), interior vertices
 *    [ng, ng+n].
 *  - Grid functions are passed as an array of device pointers indexed by
 *    axb_gf (the reference's variable names).  Pointers a call does not use
 *    may be NULL.
 */
#ifndef ASTERX_B200_H
#define ASTERX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#define AXB_EXTERN extern "C"
#else
#define AXB_EXTERN extern
#endif
#define AXB_API AXB_EXTERN __attribute__((visibility("default")))

/* ------------------------------------------------------------------------ */
/* status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum axb_status {
  AXB_OK = 0,
  AXB_ERR_ARG = 1,        /* invalid argument (null pointer, bad size/enum) */
  AXB_ERR_GHOSTS = 2,     /* too few ghost layers for the stencil            */
  AXB_ERR_CUDA = 3,       /* a CUDA runtime call failed                      */
  AXB_ERR_UNSUPPORTED = 4,/* option combination not implemented             */
  AXB_ERR_TOO_LARGE = 5,  /* size beyond a documented limit                 */
  AXB_ERR_NO_DEVICE = 6   /* no usable sm_100 device                         */
} axb_status;

/* Device error-word bits (axb_error_word). */
#define AXB_EW_NAN_FLUX 0x1u   /* non-finite face flux (reference asserts)   */
#define AXB_EW_NAN_RHS 0x2u    /* non-finite hydro RHS (rhs.cxx:199-206)      */
#define AXB_EW_C2P_FAIL 0x4u   /* at least one cell ended as C2P_FAIL        */
#define AXB_EW_ROOT_CAP 0x8u   /* an EOS temperature root find hit its cap    */
#define AXB_EW_QUEUE_TIMEOUT 0x10u /* persistent work queue gave up          */
#define AXB_EW_MMA_TIMEOUT 0x20u /* a tensor-core wait of the learned guess gave up */

/* ------------------------------------------------------------------------ */
/* grid functions                                                            */
/* ------------------------------------------------------------------------ */
#define AXB_GF_LIST(X)                                                         \
  /* ADMBaseX, vertex-centred */                                               \
  X(gxx) X(gxy) X(gxz) X(gyy) X(gyz) X(gzz) X(alp) X(betax) X(betay) X(betaz)  \
  X(kxx) X(kxy) X(kxz) X(kyy) X(kyz) X(kzz)                                    \
  /* HydroBaseX primitives, cell-centred */                                    \
  X(rho) X(velx) X(vely) X(velz) X(eps) X(press) X(temperature) X(Ye)          \
  X(entropy) X(Bvecx) X(Bvecy) X(Bvecz)                                        \
  /* conserved variables and their RHS, cell-centred */                        \
  X(dens) X(momx) X(momy) X(momz) X(tau) X(DYe) X(DEnt)                        \
  X(densrhs) X(momxrhs) X(momyrhs) X(momzrhs) X(taurhs) X(DYe_rhs) X(DEntrhs)  \
  /* vector potential (edges) and Psi (vertices) and their RHS */              \
  X(Avec_x) X(Avec_y) X(Avec_z) X(Psi)                                         \
  X(Avec_x_rhs) X(Avec_y_rhs) X(Avec_z_rhs) X(Psi_rhs)                         \
  /* staggered and centred densitised magnetic field */                        \
  X(dBx_stag) X(dBy_stag) X(dBz_stag) X(dBx) X(dBy) X(dBz)                     \
  /* con2prim bookkeeping, cell-centred */                                     \
  X(con2prim_flag) X(saved_rho) X(saved_velx) X(saved_vely) X(saved_velz)      \
  X(saved_eps) X(saved_Ye)                                                     \
  X(zvec_x) X(zvec_y) X(zvec_z) X(svec_x) X(svec_y) X(svec_z)                  \
  /* scratch: vertex auxiliaries of the A/Psi RHS (fluxes.cxx:798-826) */      \
  X(Fx) X(Fy) X(Fz) X(Fbetax) X(Fbetay) X(Fbetaz) X(G)                         \
  /* scratch: face fluxes of the transverse B components (rhs.cxx:171-172) */  \
  X(fxBy) X(fxBz) X(fyBx) X(fyBz) X(fzBx) X(fzBy)                              \
  /* scratch: partial flux divergence of the 7 hydro variables */              \
  X(acc_dens) X(acc_momx) X(acc_momy) X(acc_momz) X(acc_tau) X(acc_DYe)        \
  X(acc_DEnt)                                                                  \
  /* upwind CT face data (use_uct; AsterX/interface.ccl:135-165): the  */      \
  /* transverse vtilde^i = alpha v^i - beta^i averaged with the bounding */    \
  /* speeds, and those speeds amax, amin, per face direction */                \
  X(vtilde_y_xface) X(vtilde_z_xface) X(vtilde_z_yface) X(vtilde_x_yface)      \
  X(vtilde_x_zface) X(vtilde_y_zface) X(amax_xface) X(amin_xface)              \
  X(amax_yface) X(amin_yface) X(amax_zface) X(amin_zface)

typedef enum axb_gf {
#define AXB_GF_ENUM_(name) AXB_GF_##name,
  AXB_GF_LIST(AXB_GF_ENUM_)
#undef AXB_GF_ENUM_
  AXB_NUM_GF
} axb_gf;

typedef struct axb_box {
  int32_t n[3];      /* interior cells per axis                           */
  int32_t ng;        /* ghost layers per axis (>= 3)                       */
  int64_t sy, sz;    /* element strides of j and k (stride of i is 1)      */
  double dx[3];      /* grid spacing                                       */
  double xmin[3];    /* coordinate of vertex (ng, ng, ng)                  */
} axb_box;

typedef struct axb_fields {
  double *gf[AXB_NUM_GF];
} axb_fields;

/* ------------------------------------------------------------------------ */
/* parameters: the param.ccl keywords of AsterX, ReconX and Con2PrimFactory */
/* ------------------------------------------------------------------------ */
typedef enum axb_recon {
  AXB_RECON_GODUNOV = 0,
  AXB_RECON_MINMOD = 1,
  AXB_RECON_MONOCENTRAL = 2,
  AXB_RECON_PPM = 3,
  AXB_RECON_EPPM = 4,
  AXB_RECON_WENOZ = 5,
  AXB_RECON_MP5 = 6
} axb_recon;
typedef enum axb_flux { AXB_FLUX_LXF = 0, AXB_FLUX_HLLE = 1 } axb_flux;
typedef enum axb_recvar { AXB_RECVAR_V = 0, AXB_RECVAR_Z = 1, AXB_RECVAR_S = 2 } axb_recvar;
typedef enum axb_gauge { AXB_GAUGE_ALGEBRAIC = 0, AXB_GAUGE_GEN_LORENZ = 1 } axb_gauge;
typedef enum axb_c2p {
  AXB_C2P_NONE = 0,
  AXB_C2P_NOBLE = 1,
  AXB_C2P_PALENZUELA = 2,
  AXB_C2P_ENTROPY = 3
} axb_c2p;

/* c2p cell flags, identical to AsterX/src/con2prim.cxx:27-35 */
typedef enum axb_c2p_flag {
  AXB_C2P_INIT = 0,
  AXB_C2P_PRIME = 1,
  AXB_C2P_SECOND = 2,
  AXB_C2P_ENTROPY_OK = 3,
  AXB_C2P_ATMO = 4,
  AXB_C2P_AVG = 5,
  AXB_C2P_FAIL = 6
} axb_c2p_flag;

typedef struct axb_params {
  /* ReconX (ReconX/param.ccl) */
  int32_t reconstruction_method;   /* axb_recon, default GODUNOV          */
  int32_t loworder_method;         /* GODUNOV | MINMOD | MONOCENTRAL      */
  int32_t reconstruct_with_temperature;
  int32_t ppm_shock_detection, ppm_zone_flattening;
  double ppm_eta1, ppm_eta2, ppm_eps, ppm_eps_shock, ppm_small, ppm_omega1,
      ppm_omega2, enhanced_ppm_C2, weno_eps, mp5_alpha;
  /* EOSX polytrope used by PPM shock detection (EOSX/param.ccl:22-30) */
  double poly_k, poly_gamma;
  /* AsterX (AsterX/param.ccl) */
  int32_t flux_type;               /* axb_flux, default LXF               */
  int32_t recon_type;              /* axb_recvar, default V               */
  int32_t vector_potential_gauge;  /* axb_gauge, default GEN_LORENZ       */
  int32_t local_spatial_order;     /* 2 or 4                              */
  int32_t use_uct, use_entropy_fix, excise, use_mask;
  double lorenz_damp_fac;
  /* Con2PrimFactory (Con2PrimFactory/param.ccl) */
  int32_t c2p_prime, c2p_second;   /* axb_c2p                             */
  int32_t max_iter;
  int32_t thermal_eos_atmo, use_press_atmo, use_z, use_temperature,
      Ye_lenient;
  double c2p_tol, rho_abs_min, atmo_tol, eps_atmo, p_atmo, t_atmo, Ye_atmo,
      r_atmo, n_rho_atmo, n_press_atmo, n_temp_atmo, alp_thresh, rho_BH,
      eps_BH, vwlim_BH, cons_error_limit, vw_lim, B_lim;
} axb_params;

/* Fill p with the reference defaults of every param.ccl above. */
AXB_API void axb_params_default(axb_params *p);

/* Name of grid function `id` (the reference's variable name), NULL if out of
 * range. */
AXB_API const char *axb_gf_name(int id);

/* ------------------------------------------------------------------------ */
/* context and device status                                                 */
/* ------------------------------------------------------------------------ */
typedef struct axb_ctx axb_ctx;

/* Bind to CUDA device `device` (must be sm_100) and allocate the small
 * device status block (error word, CFL maximum, c2p counters) and a second
 * stream with three events, onto which the RHS group forks the kernels that
 * do not depend on the flux passes (joined back into the caller's stream
 * before the call's last kernel).  A context serves one host thread at a
 * time; give each thread its own.  No counterpart in the reference, whose
 * device errors are asserts. */
AXB_API int axb_ctx_create(int device, axb_ctx **out);
AXB_API int axb_ctx_destroy(axb_ctx *ctx);

/* Zero the status block, stream-ordered. */
AXB_API int axb_status_reset(axb_ctx *ctx, void *stream);

/* Synchronise `stream` and read the status block: error word (AXB_EW_*),
 * the maximum characteristic speed max|lambda| over all faces of the flux
 * passes since the last reset (the CFL input; the reference keeps per-face
 * amax/amin instead, AsterX/src/fluxes.cxx:779-785), the number of cells
 * that ended as C2P_FAIL, and a 64-bin histogram of first-solver iteration
 * counts.  Any output pointer may be NULL. */
AXB_API int axb_status_read(axb_ctx *ctx, void *stream, uint32_t *error_word,
                            double *max_speed, uint32_t *c2p_fail,
                            uint64_t *iter_hist64);

/* ------------------------------------------------------------------------ */
/* equations of state                                                        */
/* ------------------------------------------------------------------------ */
typedef struct axb_eos axb_eos;

/* Ideal gas p = (Gamma-1) rho eps with validity ranges, as EOSX_Setup_EOS
 * builds eos_3p_idealgas (EOSX/src/setup_eos.cxx:70-78,
 * EOSX/src/eos_3p_idealgas/eos_3p_idealgas.hxx:124-142), plus the
 * initial-data polytrope (poly_gamma, poly_k) the cold atmosphere uses
 * (EOSX/src/setup_eos.cxx:33-41).  Host-only; allocates nothing on the
 * device. */
AXB_API int axb_eos_create_idealgas(double gamma, double particle_mass,
                                    const double rho_range[2],
                                    const double eps_range[2],
                                    const double ye_range[2], double poly_gamma,
                                    double poly_k, axb_eos **out);

/* Tabulated3d EOS (eos_3p_tabulated3d) from a table already read and
 * converted, in the state eos_3p_tabulated3d::init leaves it
 * (EOSX/src/eos_3p_tabulated3d/eos_3p_tabulated3d.hxx:53-192; the HDF5 read
 * itself stays with the caller): uniform axes logrho[nrho] and logtemp[ntemp]
 * (natural logs), ye[nye], and `table` holding 19 variables per node,
 * variable fastest, node = i_rho + nrho * (i_temp + ntemp * i_ye); variables
 * 0 (ln press), 1 (ln(eps + energy_shift)), 2 (entropy) and 4 (cs^2) are
 * used.  Ranges as at the end of init (:179-192).  Copies the four used
 * variables to the current device (one cudaMalloc; 32 B per node).  The
 * fluxes need reconstruct_with_temperature = 1 with this EOS, as in the
 * reference.  Temperature inversions are capped at 10000 Brent steps
 * (AXB_EW_ROOT_CAP). */
AXB_API int axb_eos_create_tabulated3d(int nrho, int ntemp, int nye,
                                       const double *logrho, const double *logtemp,
                                       const double *ye, const double *table,
                                       double energy_shift, double poly_gamma,
                                       double poly_k, axb_eos **out);
/* StellarCollapse tables (eos_3p_tabulated3d::init,
 * EOSX/src/eos_3p_tabulated3d/eos_3p_tabulated3d.hxx:53-193), from the
 * datasets the caller read from the HDF5 file (no HDF5 library is linked):
 * logrho10[nrho], logtemp10[ntemp] (log10 of g/cm^3 and MeV), ye_in[nye],
 * energy_shift_cgs (erg/g), and dsets[19] = "logpress", "logenergy",
 * "entropy", "munu", "cs2", "dedt", "dpdrhoe", "dpderho", "muhat", "mu_e",
 * "mu_p", "mu_n", "Xa", "Xh", "Xn", "Xp", "Abar", "Zbar", "gamma", each
 * nrho*ntemp*nye values with rho fastest, as stored in the file.
 *
 * axb_eos_stellarcollapse_convert applies init's conversions
 * (:115-177): natural logs in code units (EOSX/src/utils/
 * eos_constants.hxx:7-14), cs^2 and the derivatives scaled, the 19
 * variables interleaved per node -- the arguments of
 * axb_eos_create_tabulated3d: logrho, logtemp, ye (nrho, ntemp, nye values),
 * table (19 * nrho * ntemp * nye), energy_shift; and, if `ranges` is not
 * NULL, the ranges init sets (:179-192): rho min/max, temperature min/max,
 * Ye min/max, eps min/max.  Host only; allocates nothing.
 * axb_eos_create_stellarcollapse converts and then calls
 * axb_eos_create_tabulated3d. */
AXB_API int axb_eos_stellarcollapse_convert(int nrho, int ntemp, int nye,
                                            const double *logrho10, const double *logtemp10,
                                            const double *ye_in, const double *const *dsets,
                                            double energy_shift_cgs, double *logrho,
                                            double *logtemp, double *ye, double *table,
                                            double *energy_shift, double ranges[8]);
AXB_API int axb_eos_create_stellarcollapse(int nrho, int ntemp, int nye,
                                           const double *logrho10, const double *logtemp10,
                                           const double *ye_in, const double *const *dsets,
                                           double energy_shift_cgs, double poly_gamma,
                                           double poly_k, axb_eos **out);
AXB_API int axb_eos_destroy(axb_eos *eos);

/* ------------------------------------------------------------------------ */
/* scheduled routines                                                        */
/* ------------------------------------------------------------------------ */

/* AsterX_RHSGroup on one box (AsterX/schedule.ccl:169-228), replacing the
 * scheduled routines AsterX_Fluxes (AsterX/src/fluxes.cxx:828-878),
 * AsterX_SourceTerms (AsterX/src/source.cxx:170-185) and AsterX_RHS
 * (AsterX/src/rhs.cxx:18-253).
 * Reads: ADMBaseX metric, lapse, shift, curvature; HydroBaseX primitives;
 *   dB*_stag; Avec_*; Psi -- on the interior and ng ghost layers.
 * Writes: densrhs .. DEntrhs (interior cells), Avec_*_rhs (interior edges),
 *   Psi_rhs (interior vertices).
 * Scratch: acc_*, fxBy .. fzBy, Fx .. G.
 * Face quantities the reference obtains by SYNC (face B fluxes one cell
 * outside the interior, vertex auxiliaries two vertices outside) are computed
 * from the ghost data instead, so no synchronisation is needed inside the
 * group.  Requires ng >= 3; recon_type v_vec, z_vec (zvec_*) or s_vec
 * (svec_*).  With use_uct (upwind CT, rhs.cxx:124-168) the fields also hold
 * the twelve face arrays vtilde_*face, amax_*face, amin_*face (written), the
 * face data are computed three layers outside the interior, and dB*_stag
 * must be valid on three ghost layers.  The CFL speed maximum accumulates
 * into the context status. */
AXB_API int axb_rhs_group(axb_ctx *ctx, const axb_box *box,
                          const axb_fields *fields, const axb_params *params,
                          const axb_eos *eos, void *stream);

/* AsterX_Con2PrimGroup on one box (AsterX/schedule.ccl:119-165), replacing
 * AsterX_ComputedBstagFromA (AsterX/src/computeBfromA.cxx:58-65),
 * AsterX_ComputedBFromdBstag (:67-85) and AsterX_Con2Prim
 * (AsterX/src/con2prim.cxx:457-502) with the Con2PrimFactory functors
 * c2p_2DNoble::solve (Con2PrimFactory/src/c2p_2DNoble.hxx:275-594),
 * c2p_1DPalenzuela::solve (Con2PrimFactory/src/c2p_1DPalenzuela.hxx:306-556)
 * and c2p_1DEntropy::solve (Con2PrimFactory/src/c2p_1DEntropy.hxx:306-469).
 * Reads: Avec_* (interior edges + one ghost layer), conserved variables,
 *   saved_* and temperature (seeds), metric and lapse.
 * Writes: dB*_stag on the interior faces and one transverse ghost layer,
 *   dB*, the HydroBaseX primitives, conserved variables (after floors),
 *   saved_*, con2prim_flag, and zvec_* / svec_* when given.
 * c2p_prime and c2p_second are Noble, Palenzuela or Entropy (second may be
 * None); use_entropy_fix runs the entropy scheme on cells both failed
 * (flag AXB_C2P_ENTROPY_OK when it recovers them).  The entropy scheme
 * needs the ideal gas (a table defines no p(rho, kappa)); use_mask is not
 * supported (AXB_ERR_UNSUPPORTED).
 * C2P_FAIL cells are counted in the context status. */
AXB_API int axb_con2prim_group(axb_ctx *ctx, const axb_box *box,
                               const axb_fields *fields,
                               const axb_params *params, const axb_eos *eos,
                               void *stream);

/* One Runge-Kutta stage of the 11 evolved variables (dens, mom*, tau, DYe,
 * DEnt, Avec_*, Psi) on their interiors:
 *   out = alpha * U_n + beta * U_k + gamma * dt * RHS.
 * This is the stage combine that CarpetX's ODESolvers performs around the
 * reference's scheduled routines (no counterpart in the reference sources);
 * SSP-RK3 in Shu-Osher form uses (0,1,1), (3/4,1/4,1/4), (1/3,2/3,2/3).
 * `out`, `un` and `uk` may be the same fields. */
AXB_API int axb_rk_stage(axb_ctx *ctx, const axb_box *box, const axb_fields *out,
                         const axb_fields *un, const axb_fields *uk,
                         const axb_fields *rhs, double alpha, double beta,
                         double gamma, double dt, void *stream);

/* Periodic ghost fill of the grid functions `ids[0..nids)` of one box, each
 * with its own centring: the single-box form of the driver's SYNC with
 * periodic outer boundaries (AsterX/schedule.ccl:110-115,157-164). */
AXB_API int axb_sync_periodic(axb_ctx *ctx, const axb_box *box,
                              const axb_fields *fields, const int *ids, int nids,
                              void *stream);

/* ------------------------------------------------------------------------ */
/* grid functions in the caller's own per-centring layouts                   */
/* ------------------------------------------------------------------------ */

/* A set of grid functions each with its own j and k strides: gf[id] points at
 * the field's point (0, 0, 0) (the first ghost point of the box in every
 * direction) and holds its centring's n[d] + 2*ng (cell) or n[d] + 2*ng + 1
 * (vertex) points per direction at f[i + sy[id]*j + sz[id]*k] -- the layout
 * CarpetX gives each centring of a box (a cell-centred field one point
 * shorter per cell direction than a vertex-centred one).  No counterpart in
 * the reference, whose GF3D2 views carry these strides per field. */
typedef struct axb_fields_strided {
  double *gf[AXB_NUM_GF];
  int64_t sy[AXB_NUM_GF], sz[AXB_NUM_GF];
} axb_fields_strided;

/* Copy the grid functions ids[0..nids) of `src` (per-field strides) into
 * the engine's layout of `box` (`dst`, strides box->sy, box->sz), every
 * point of each field's centring, ghosts included; axb_export_fields copies
 * back.  A caller whose fields are laid out per centring wraps the engine's
 * groups with these copies (one read and one write per point). */
AXB_API int axb_import_fields(axb_ctx *ctx, const axb_box *box,
                              const axb_fields_strided *src, const int *ids, int nids,
                              const axb_fields *dst, void *stream);
AXB_API int axb_export_fields(axb_ctx *ctx, const axb_box *box, const axb_fields *src,
                              const int *ids, int nids, const axb_fields_strided *dst,
                              void *stream);

/* ------------------------------------------------------------------------ */
/* physical outer boundaries and general Runge-Kutta methods                 */
/* ------------------------------------------------------------------------ */

/* Outer-boundary rules of CarpetX's boundary_x .. boundary_upper_z
 * parameters that the reference's tests use (AsterX/test/*.par). */
typedef enum axb_bc {
  AXB_BC_PERIODIC = 0, /* ghost = periodic image                          */
  AXB_BC_NEUMANN = 1,  /* "neumann": ghost = outermost interior point      */
  AXB_BC_LINEAR = 2    /* "linear extrapolation" from the two outermost
                          interior points                                   */
} axb_bc;

/* Fill the ghost layers of the grid functions ids[0..nids), each with its
 * own centring, by the rule of each face: bc[0..5] = x-lower, x-upper,
 * y-lower, y-upper, z-lower, z-upper; the x ghosts first (over all y, z
 * points), then y, then z, so edges and corners take each direction's rule
 * in turn.  The boundary point of a face is the outermost interior point of
 * the centring (the boundary vertex itself for a vertex-centred direction).
 * The driver applies this on every SYNC of a grid function with a physical
 * boundary (AsterX/schedule.ccl's SYNC lists); no counterpart in the
 * reference sources. */
AXB_API int axb_fill_boundary(axb_ctx *ctx, const axb_box *box, const axb_fields *fields,
                              const int *ids, int nids, const int bc[6], void *stream);

/* axb_rhs_group for a box with the outer-boundary rules bc[6]: the face B
 * fluxes (fxBy .. fzBy) and the vertex auxiliaries (Fx .. G) are computed on
 * the interior and then filled on the ghost points by axb_fill_boundary, as
 * the reference's AsterX_Fluxes writes them on the interior and SYNCs them
 * (AsterX/schedule.ccl:174-195); axb_rhs_group instead computes them from
 * the ghost data, which equals this when every face is periodic. */
AXB_API int axb_rhs_group_bc(axb_ctx *ctx, const axb_box *box, const axb_fields *fields,
                             const axb_params *params, const axb_eos *eos,
                             const int bc[6], void *stream);

/* The general stage combination of an explicit Runge-Kutta method on the
 * interiors of the 11 evolved variables:
 *   out = sum_{q < nstates} coef[q] * states[q] + gdt * RHS,   nstates <= 4,
 * as CarpetX's ODESolvers forms its stages (RK2, RK3, RK4 with their
 * stored stages).  `out` may be one of the states; `rhs` holds the RHS grid
 * functions (densrhs .. Psi_rhs).  No counterpart in the reference
 * sources. */
AXB_API int axb_rk_lincomb(axb_ctx *ctx, const axb_box *box, const axb_fields *out,
                           int nstates, const double *coef,
                           const axb_fields *const *states, double gdt,
                           const axb_fields *rhs, void *stream);

/* One RK substep of one box: axb_rhs_group with axb_rk_stage fused into its
 * last kernels (U_k updated in place in `fields`, U_n read from `fields_n`;
 * the RHS grid functions are not written), periodic fill of the evolved
 * variables (if `periodic`), axb_con2prim_group, periodic fill of the
 * primitives and of zvec / svec when recon_type reconstructs them (if
 * `periodic`).  Stream-ordered, allocation-free. */
AXB_API int axb_substep(axb_ctx *ctx, const axb_box *box,
                        const axb_fields *fields, const axb_fields *fields_n,
                        const axb_params *params, const axb_eos *eos,
                        double alpha, double beta, double gamma, double dt,
                        int periodic, void *stream);

/* ------------------------------------------------------------------------ */
/* batched substep over the boxes of a refinement level                      */
/* ------------------------------------------------------------------------ */

/* A level of boxes advanced together.  CarpetX runs each scheduled routine
 * of AsterX_RHSGroup and AsterX_Con2PrimGroup (AsterX/schedule.ccl:119-228)
 * as one loop launch per box; a batch runs each phase of the substep as ONE
 * persistent launch over the tiles of all its boxes, with results
 * bit-identical to axb_substep on every box.  axb_batch_create checks every
 * box as axb_rhs_group / axb_con2prim_group would, copies the per-box
 * argument blocks and tile tables to the device (its only allocations), and
 * keeps `eos` by reference: it must outlive the batch.  Field pointers are
 * fixed at creation (U_k in fields[b], U_n in fields_n[b]). */
typedef struct axb_batch axb_batch;
AXB_API int axb_batch_create(axb_ctx *ctx, int nbox, const axb_box *boxes,
                             const axb_fields *fields, const axb_fields *fields_n,
                             const axb_params *params, const axb_eos *eos,
                             axb_batch **out);
AXB_API int axb_batch_destroy(axb_batch *batch);

/* One RK substep of every box (axb_substep semantics), as 12 stream-ordered
 * launches and one memset, allocation-free: a caller may capture it in a
 * CUDA graph. */
AXB_API int axb_batch_substep(axb_ctx *ctx, axb_batch *batch, double alpha,
                              double beta, double gamma, double dt, int periodic,
                              void *stream);

/* Autotuner: times the RHS phases on the batch's own boxes for pencil
 * segments {8, 16, 32, 64} of the y and z flux passes and persistent grids
 * of {2, 4, 8, 16} CTAs per SM, and keeps the fastest.  Leaves the RHS grid
 * functions as one RHS evaluation would.  Synchronous; not for use inside a
 * stream capture.  out (may be NULL, 3 ints): y segment, z segment, CTAs per
 * SM of the flux passes.  No counterpart in the reference. */
AXB_API int axb_batch_autotune(axb_ctx *ctx, axb_batch *batch, int *out, void *stream);

/* ------------------------------------------------------------------------ */
/* independent-cell primitive recovery and the learned initial guess         */
/* ------------------------------------------------------------------------ */

/* Structure-of-arrays view of `n` independent cells (device pointers, one
 * double per cell each).  Conserved variables are densitized as the
 * reference's cons_vars (Con2PrimFactory/src/cons.hxx:48-91): dens, mom_i,
 * tau, DYe, DEnt, dB^i; g holds the cell's gamma_ij (xx xy xz yy yz zz).
 * Seeds (saved primitives: rho, eps, Ye, vel^i, temperature) may all be NULL
 * for a cold start: v = 0, eps = the atmosphere's eps, Ye = DYe/dens.
 * Outputs (any may be NULL): rho, eps, press, vel^i, w_lorentz, Ye,
 * temperature, entropy, the iteration count of the first solver (double;
 * with a learned guess that failed, its attempt and the cold-start retry
 * together), the con2prim flag (AXB_C2P_* code, as double), and with a
 * learned guess `fallback` (1 where the guessed first attempt failed and the
 * plain cascade recovered or failed the cell, else 0). */
typedef struct axb_cells {
  int64_t n;
  const double *dens, *mom[3], *tau, *DYe, *DEnt, *dB[3];
  const double *g[6];
  const double *seed_rho, *seed_eps, *seed_Ye, *seed_vel[3], *seed_temperature;
  double *rho, *eps, *press, *vel[3], *w_lorentz, *Ye, *temperature, *entropy;
  double *iters, *flag;
  float *guess;     /* scratch, 2 floats per cell; required with a learned guess */
  double *fallback; /* output, may be NULL */
} axb_cells;

/* Learned initial guess: an MLP nf -> 64 -> 64 -> 64 -> 2 (SiLU or ReLU
 * hidden activations; nf = 8, or 9 with Ye for a tabulated EOS) evaluated in
 * BF16 on the tensor cores (tcgen05, tiles of 128 cells, FP32 accumulators in
 * tensor memory).
 * Outputs: y0 = the position of x = h W in the Palenzuela scheme's
 * initial bracket [max(1e-10, 1 + q - s), 2 + 2 q - s]
 * (c2p_1DPalenzuela.hxx:395-398), y1 = ln W.  The Noble scheme starts from
 * Z = D x and v^2 = 1 - W^-2 instead of its saved-primitive seeds
 * (c2p_2DNoble.hxx:374-393), the Palenzuela scheme brackets x by
 * [x (1 - bracket), x (1 + bracket)] when that interval brackets the root
 * and otherwise keeps its own bracket (c2p_1DPalenzuela.hxx:395-401).
 * The network runs in its own kernel before the recovery (a persistent
 * grid whose CTAs stage the weights in shared memory once) and leaves
 * (x, W) per cell in the caller's `guess` scratch.  A cell whose guessed
 * first attempt fails is
 * retried from the plain cold-start seeds of c2p_2DNoble.hxx:374-393 (and
 * the plain bracket) before the second scheme, so the cascade after a
 * failed guess is exactly the plain one.
 * No counterpart in the reference. */
typedef struct axb_mlp axb_mlp;

#define AXB_MLP_HIDDEN 64
#define AXB_MLP_MAXF 16

/* Number of parameters of an MLP with `nf` inputs:
 * W1 [nf x 64], b1 [64], W2 [64 x 64], b2, W3 [64 x 64], b3, W4 [64 x 2], b4 [2]
 * in that order, row-major (input index outer). */
AXB_API int64_t axb_mlp_param_count(int nf);

/* Create an MLP on the current device from FP32 parameters (host memory, in
 * the order above), or with seeded random initial values when `params` is
 * NULL.  `bracket` is the relative half-width of the Palenzuela bracket. */
AXB_API int axb_mlp_create(int nf, const float *params, uint64_t seed,
                           double bracket, axb_mlp **out);

/* Hidden activations of the network. */
#define AXB_MLP_SILU 0 /* z sigmoid(z) (axb_mlp_create's choice)           */
#define AXB_MLP_RELU 1 /* max(z, 0): no special-function instruction       */

/* axb_mlp_create with the hidden activation chosen (AXB_MLP_SILU or
 * AXB_MLP_RELU); training and inference use it alike. */
AXB_API int axb_mlp_create_act(int nf, int activation, const float *params,
                               uint64_t seed, double bracket, axb_mlp **out);
AXB_API int axb_mlp_destroy(axb_mlp *mlp);
/* Copy the FP32 master parameters to host memory (param_count floats). */
AXB_API int axb_mlp_get_params(const axb_mlp *mlp, float *params);

/* The MLP input features of each cell (n x nf FP32, row-major, device), as
 * the recovery kernel computes them: with sqrt(gamma)-undensitized D, S_i,
 * tau, B^i and q = tau/D, r = S^2/D^2, s = B^2/D, t = B.S/D^1.5:
 * ln D / 10, ln(1+q), ln(1+r)/2, ln(1+s), t^2/(r s), r/(1+q+s)^2, s/(1+q+s),
 * ln(1+q) - ln(1+r)/2 [, Ye = DYe/dens]. */
AXB_API int axb_mlp_features(axb_ctx *ctx, const axb_cells *cells, int nf,
                             float *features, void *stream);

/* The network's outputs (n x 2 FP32, device) for given features (n x nf
 * FP32, device), through the same tensor-core code the recovery kernel
 * runs. */
AXB_API int axb_mlp_forward(axb_ctx *ctx, const axb_mlp *mlp, const float *features,
                            int64_t n, float *out, void *stream);

/* One optimisation step on a batch: forward with BF16-rounded weights and
 * activations (as the tensor-core inference sees them) and FP32 accumulation,
 * mean-squared error against `targets` (n x 2 FP32, device), backward in
 * FP32, Adam (lr, beta1, beta2, eps) on the FP32 master parameters.  The
 * batch loss is written to `loss` (device FP32, may be NULL).  If `grad` is
 * non-NULL the parameter gradient (param_count floats, device) is written
 * there and no update is made. */
AXB_API int axb_mlp_train_step(axb_ctx *ctx, axb_mlp *mlp, const float *features,
                               const float *targets, int64_t n, float lr,
                               float beta1, float beta2, float adam_eps,
                               float *loss, float *grad, void *stream);

/* The primitive recovery of AsterX_Con2Prim_typeEoS (con2prim.cxx:137-416)
 * for independent cells: cons floors, the c2p_prime -> c2p_second cascade
 * with atmosphere on double failure, and a uniform atmosphere built from
 * `params` (rho_abs_min etc., as for a box inside r_atmo).  With `mlp`
 * non-NULL the learned guess replaces the seeds as described above.  The
 * iteration histogram and failure count accumulate into the context status.
 * No mask/excision. */
AXB_API int axb_c2p_cells(axb_ctx *ctx, const axb_cells *cells,
                          const axb_params *params, const axb_eos *eos,
                          const axb_mlp *mlp, void *stream);

/* axb_con2prim_group with the learned guess of the first solver: after
 * curl A, the network evaluates every interior cell (its conserved variables,
 * the cell average of dB_stag, the metric averaged from the eight vertices),
 * and the first solver starts from that guess (Noble's seeds or the
 * Palenzuela bracket, as above); a cell whose guessed first attempt fails is
 * recovered again from the plain seeds (saved_*) through the plain cascade.
 * The tabulated EOS needs a 9-input network (Ye).  The first solver's
 * iterations of both attempts count in the context's histogram.  Uses a
 * scratch float2 per interior cell from the stream-ordered allocator.
 * `mlp` must be non-NULL (AXB_ERR_ARG).  No counterpart in the reference. */
AXB_API int axb_con2prim_group_guess(axb_ctx *ctx, const axb_box *box,
                                     const axb_fields *fields, const axb_params *params,
                                     const axb_eos *eos, const axb_mlp *mlp, void *stream);

/* axb_rhs_group for callers that cannot allocate device memory (a host
 * framework that owns every device allocation, a tool that may not call
 * cudaMalloc on a shared device, a driver whose footprint is fixed after
 * set-up).  No counterpart in the reference.  Inputs and outputs are as for
 * axb_rhs_group; the 20 scratch grid functions (acc_*, fxBy..fzBy, Fx..G) are
 * ignored if given and taken instead from a 16 MiB array that this library
 * holds in static device memory on every GPU it is loaded on, until exit.
 * Limit: 20 * sz * (n[2] + 2*ng + 1) doubles (each of the 20 rounded up to
 * 32) must fit in 2^21 doubles; the limit is that formula, so it depends on
 * the caller's row and plane padding (sy, sz) -- for example a 32^3 box with
 * 3 ghosts and rows padded to 4 doubles fits, a 48^3 box does not.  Larger
 * boxes get AXB_ERR_TOO_LARGE, and n[d] or ng outside [1, 2^15] (ng >= 3 is
 * required as for axb_rhs_group) AXB_ERR_ARG, before anything runs.  Calls
 * no cudaMalloc, cudaFree or allocating library routine and needs no
 * axb_ctx.  The device error word and the CFL maximum go to a static status
 * block that this entry point clears on every call and that is not
 * reported: a caller that needs them (for instance the root-cap flag of a
 * tabulated EOS) uses axb_rhs_group.  use_uct is not available here (its
 * twelve face arrays are not part of the static scratch).   The first call on a device looks up the
 * arrays' device addresses with that device current; make it before any
 * stream capture.  All calls share the arrays: calls that overlap on the GPU
 * (other streams, other threads) race; order them on one stream. */
AXB_API int axb_rhs_group_noalloc(const axb_box *box, const axb_fields *fields,
                                  const axb_params *params, const axb_eos *eos,
                                  void *stream);

/* ------------------------------------------------------------------------ */
/* multi-GPU: halo exchange of a z-slab decomposition over NCCL              */
/* ------------------------------------------------------------------------ */

/* The analogue of the driver's SYNC (AsterX/schedule.ccl:110-115,157-164)
 * between ranks that each hold one z-slab of a periodic patch (one process
 * per GPU; no counterpart as a routine in the reference, where CarpetX/AMReX
 * does it).  axb_halo_unique_id makes the NCCL id on one rank (the caller
 * hands it to the others); axb_halo_create builds the communicator and the
 * packed buffers for the listed grid functions of this rank's box (n[2] =
 * its slab's cells, at least ng); axb_halo_exchange replaces the ng ghost
 * k-planes below and above the slab by the neighbours' planes: one pack
 * kernel, one NCCL group of two sends and two receives, one unpack kernel,
 * all on `stream`.  Plane mapping for nz interior cells and v = 1 for a
 * field vertex-centred in z: ghosts [0, ng) <- lower neighbour's
 * [nz, nz + ng); ghosts [ng + nz + v, 2 ng + nz + v) <- upper neighbour's
 * [ng + v, 2 ng + v); with one rank this is the periodic wrap in z.  The x
 * and y ghosts are filled beforehand by axb_sync_periodic (whose z wrap the
 * exchange then overwrites). */
typedef struct axb_halo axb_halo;
AXB_API int axb_halo_unique_id(unsigned char id[128]);
AXB_API int axb_halo_create(axb_ctx *ctx, const axb_box *box, int nranks, int rank,
                            const unsigned char id[128], const int *field_ids, int nfields,
                            axb_halo **out);
AXB_API int axb_halo_exchange(axb_halo *halo, const axb_fields *fields, void *stream);
AXB_API int axb_halo_destroy(axb_halo *halo);

/* ------------------------------------------------------------------------ */
/* stress-energy tensor and regrid error                                     */
/* ------------------------------------------------------------------------ */

/* AsterX_Tmunu (AsterX/src/tmunu.cxx:19-178, scheduled in
 * TmunuBaseX_AddToTmunu): at every interior vertex, the cell-centred rho,
 * eps, press, Bvec and velocity (velx.. for recon_type v_vec, zvec_x.. for
 * z_vec and s_vec, as the reference tests recon_type == "v_vec") are
 * interpolated to the vertex (interp_order 2: the mean of the 8 cells
 * around it; 4: cubic Lagrange weights over 4 cells per direction, needs 2
 * ghost layers; AsterUtils/src/aster_interp.hxx:97-148), and the ideal-MHD
 * T_{mu nu} is ADDED to eT[0..9] = eTtt, eTtx, eTty, eTtz, eTxx, eTxy,
 * eTxz, eTyy, eTyz, eTzz (vertex-centred arrays in the box's layout).
 * Reads rho, eps, press, Bvec, velx or zvec, the metric, alp and beta from
 * `fields`. */
AXB_API int axb_tmunu(axb_ctx *ctx, const axb_box *box, const axb_fields *fields,
                      const axb_params *params, int interp_order, double *const eT[10],
                      void *stream);

/* Regrid error indicators (AsterX/src/estimate_error.hxx:14-86; the
 * regrid_method keywords of AsterX/param.ccl). */
typedef enum axb_regrid {
  AXB_REGRID_FIRST_DERIV = 0,       /* "first derivative"        */
  AXB_REGRID_SECOND_DERIV = 1,      /* "second derivative"       */
  AXB_REGRID_SECOND_DERIV_NORM = 2, /* "second derivative norm"  */
  AXB_REGRID_FIRST_GRAD = 3         /* "first gradient"          */
} axb_regrid;

/* AsterX_EstimateError (AsterX/src/estimate_error.cxx:70-144): at every
 * interior cell, regrid_error = the largest indicator of `method` over the
 * grid functions vars[0..nvars) (1 <= nvars <= 9, each in the box's layout,
 * any centring: the cell's own index is used, as the reference does with
 * each variable's GF3D2), with the undivided differences to the neighbours
 * +-1 along each direction; epsilon_err is the noise filter of "second
 * derivative norm". */
AXB_API int axb_estimate_error(axb_ctx *ctx, const axb_box *box, const double *const *vars,
                               int nvars, int method, double epsilon_err,
                               double *regrid_error, void *stream);

/* Optional per-launch timing: after axb_timing_begin every kernel launch of
 * the entry points above is bracketed by CUDA events on its stream;
 * axb_timing_end waits for them and returns, per kernel region (sources,
 * flux x, flux y, flux z, aux, ct+psi, rk stage, sync, bstag, c2p, c2p
 * cells, mlp, tmunu, regrid error -- `nregions` entries), the summed
 * milliseconds and launch
 * counts.  Not part of the reference; a measurement aid. */
AXB_API int axb_timing_begin(axb_ctx *ctx);
AXB_API int axb_timing_end(axb_ctx *ctx, double *ms, int *count, int nregions);

/* FP64 rates of the current device, the peaks of the engine's
 * instruction-bound kernels: out[0] = FMA TFLOP/s (2 FLOP per FMA), out[1] =
 * IEEE divisions G/s, out[2] = square roots G/s, out[3] = reciprocal square
 * roots G/s, each from independent dependency chains over a grid of 8 CTAs
 * per SM.  Synchronous; allocates a small buffer for the call.  Not part of
 * the reference; a measurement aid. */
AXB_API int axb_probe_fp64(double out[4]);

#endif /* ASTERX_B200_H */
