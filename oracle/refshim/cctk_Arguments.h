// Test infrastructure only: Cactus argument macros for the scheduled routines
// of the reference hot path.  Read-only grid functions become
// GF3D2<const double> views and written ones GF3D2<double>, following the
// READS/WRITES clauses of AsterX/schedule.ccl:123-228.
#ifndef AXREF_SHIM_CCTK_ARGUMENTS_H
#define AXREF_SHIM_CCTK_ARGUMENTS_H

#include <cctk.h>
#include <loop_device.hxx>

#include "axref_fields.h"

struct cGH {
  int iteration;
};

double *axref_field(int id);
long long axref_sy();
long long axref_sz();
const Loop::GridDescBaseDevice &axref_grid();
const CCTK_REAL *axref_delta_space();

#define CCTK_ARGUMENTS const cGH *const cctkGH
#define CCTK_PASS_CTOC cctkGH
#define CCTK_DELTA_SPACE(d) (cctk_delta_space[d])

#define AXREF_RO(name)                                                         \
  const Loop::GF3D2<const CCTK_REAL> name(axref_field(AXREF_F_##name),         \
                                          axref_sy(), axref_sz());             \
  (void)name;
#define AXREF_RW(name)                                                         \
  const Loop::GF3D2<CCTK_REAL> name(axref_field(AXREF_F_##name), axref_sy(),   \
                                    axref_sz());                               \
  (void)name;

#define AXREF_COMMON                                                           \
  const Loop::GridDescBaseDevice &grid = axref_grid();                         \
  const Loop::GridDescBaseDevice &cctk_grid = grid;                            \
  const int *const cctk_nghostzones = grid.nghostzones.data();                 \
  const int cctk_iteration = cctkGH->iteration;                                \
  const CCTK_REAL *const cctk_delta_space = axref_delta_space();               \
  (void)cctk_grid;                                                             \
  (void)cctk_nghostzones;                                                      \
  (void)cctk_iteration;                                                        \
  (void)cctk_delta_space;

#define AXREF_METRIC_RO                                                        \
  AXREF_RO(gxx) AXREF_RO(gxy) AXREF_RO(gxz) AXREF_RO(gyy) AXREF_RO(gyz)        \
  AXREF_RO(gzz) AXREF_RO(alp) AXREF_RO(betax) AXREF_RO(betay) AXREF_RO(betaz)

#define AXREF_FLUXES_RW(d)                                                     \
  AXREF_RW(f##d##dens) AXREF_RW(f##d##momx) AXREF_RW(f##d##momy)               \
  AXREF_RW(f##d##momz) AXREF_RW(f##d##tau) AXREF_RW(f##d##DYe)                 \
  AXREF_RW(f##d##DEnt) AXREF_RW(f##d##Bx) AXREF_RW(f##d##By)                   \
  AXREF_RW(f##d##Bz)
#define AXREF_FLUXES_RO(d)                                                     \
  AXREF_RO(f##d##dens) AXREF_RO(f##d##momx) AXREF_RO(f##d##momy)               \
  AXREF_RO(f##d##momz) AXREF_RO(f##d##tau) AXREF_RO(f##d##DYe)                 \
  AXREF_RO(f##d##DEnt) AXREF_RO(f##d##Bx) AXREF_RO(f##d##By)                   \
  AXREF_RO(f##d##Bz)

#define DECLARE_CCTK_ARGUMENTSX_AsterX_Fluxes                                  \
  AXREF_COMMON AXREF_METRIC_RO                                                 \
  AXREF_RO(rho) AXREF_RO(velx) AXREF_RO(vely) AXREF_RO(velz) AXREF_RO(press)   \
  AXREF_RO(eps) AXREF_RO(temperature) AXREF_RO(Ye) AXREF_RO(Bvecx)             \
  AXREF_RO(Bvecy) AXREF_RO(Bvecz) AXREF_RO(entropy) AXREF_RO(dBx_stag)         \
  AXREF_RO(dBy_stag) AXREF_RO(dBz_stag) AXREF_RO(zvec_x) AXREF_RO(zvec_y)      \
  AXREF_RO(zvec_z) AXREF_RO(svec_x) AXREF_RO(svec_y) AXREF_RO(svec_z)          \
  AXREF_RO(Avec_x) AXREF_RO(Avec_y) AXREF_RO(Avec_z) AXREF_RO(Psi)             \
  AXREF_FLUXES_RW(x) AXREF_FLUXES_RW(y) AXREF_FLUXES_RW(z)                     \
  AXREF_RW(Fx) AXREF_RW(Fy) AXREF_RW(Fz) AXREF_RW(Fbetax) AXREF_RW(Fbetay)     \
  AXREF_RW(Fbetaz) AXREF_RW(G)                                                 \
  AXREF_RW(vtilde_y_xface) AXREF_RW(vtilde_z_xface) AXREF_RW(vtilde_x_yface)   \
  AXREF_RW(vtilde_z_yface) AXREF_RW(vtilde_x_zface) AXREF_RW(vtilde_y_zface)   \
  AXREF_RW(amax_xface) AXREF_RW(amin_xface) AXREF_RW(amax_yface)               \
  AXREF_RW(amin_yface) AXREF_RW(amax_zface) AXREF_RW(amin_zface)
#define DECLARE_CCTK_ARGUMENTS_AsterX_Fluxes DECLARE_CCTK_ARGUMENTSX_AsterX_Fluxes

#define DECLARE_CCTK_ARGUMENTSX_AsterX_SourceTerms                             \
  AXREF_COMMON AXREF_METRIC_RO                                                 \
  AXREF_RO(kxx) AXREF_RO(kxy) AXREF_RO(kxz) AXREF_RO(kyy) AXREF_RO(kyz)        \
  AXREF_RO(kzz) AXREF_RO(rho) AXREF_RO(press) AXREF_RO(eps) AXREF_RO(velx)     \
  AXREF_RO(vely) AXREF_RO(velz) AXREF_RO(zvec_x) AXREF_RO(zvec_y)              \
  AXREF_RO(zvec_z) AXREF_RO(svec_x) AXREF_RO(svec_y) AXREF_RO(svec_z)          \
  AXREF_RO(Bvecx) AXREF_RO(Bvecy) AXREF_RO(Bvecz)                              \
  AXREF_RW(densrhs) AXREF_RW(taurhs) AXREF_RW(momxrhs) AXREF_RW(momyrhs)       \
  AXREF_RW(momzrhs) AXREF_RW(DEntrhs) AXREF_RW(DYe_rhs)

#define DECLARE_CCTK_ARGUMENTSX_AsterX_RHS                                     \
  AXREF_COMMON AXREF_METRIC_RO                                                 \
  AXREF_RO(velx) AXREF_RO(vely) AXREF_RO(velz) AXREF_RO(press)                 \
  AXREF_FLUXES_RO(x) AXREF_FLUXES_RO(y) AXREF_FLUXES_RO(z)                     \
  AXREF_RW(densrhs) AXREF_RW(taurhs) AXREF_RW(momxrhs) AXREF_RW(momyrhs)       \
  AXREF_RW(momzrhs) AXREF_RW(DEntrhs) AXREF_RW(DYe_rhs)                        \
  AXREF_RO(Psi) AXREF_RO(Fx) AXREF_RO(Fy) AXREF_RO(Fz) AXREF_RO(Fbetax)        \
  AXREF_RO(Fbetay) AXREF_RO(Fbetaz) AXREF_RO(G) AXREF_RO(dBx_stag)             \
  AXREF_RO(dBy_stag) AXREF_RO(dBz_stag)                                        \
  AXREF_RO(vtilde_y_xface) AXREF_RO(vtilde_z_xface) AXREF_RO(vtilde_x_yface)   \
  AXREF_RO(vtilde_z_yface) AXREF_RO(vtilde_x_zface) AXREF_RO(vtilde_y_zface)   \
  AXREF_RO(amax_xface) AXREF_RO(amin_xface) AXREF_RO(amax_yface)               \
  AXREF_RO(amin_yface) AXREF_RO(amax_zface) AXREF_RO(amin_zface)               \
  AXREF_RW(Avec_x_rhs) AXREF_RW(Avec_y_rhs) AXREF_RW(Avec_z_rhs)               \
  AXREF_RW(Psi_rhs)

#define DECLARE_CCTK_ARGUMENTSX_AsterX_Tmunu                                   \
  AXREF_COMMON AXREF_METRIC_RO                                                 \
  AXREF_RO(rho) AXREF_RO(eps) AXREF_RO(press) AXREF_RO(velx) AXREF_RO(vely)    \
  AXREF_RO(velz) AXREF_RO(zvec_x) AXREF_RO(zvec_y) AXREF_RO(zvec_z)            \
  AXREF_RO(Bvecx) AXREF_RO(Bvecy) AXREF_RO(Bvecz)                              \
  AXREF_RW(eTtt) AXREF_RW(eTtx) AXREF_RW(eTty) AXREF_RW(eTtz) AXREF_RW(eTxx)   \
  AXREF_RW(eTxy) AXREF_RW(eTxz) AXREF_RW(eTyy) AXREF_RW(eTyz) AXREF_RW(eTzz)

#define DECLARE_CCTK_ARGUMENTSX_AsterX_ComputedBstagFromA                      \
  AXREF_COMMON AXREF_RO(Avec_x) AXREF_RO(Avec_y) AXREF_RO(Avec_z)              \
  AXREF_RW(dBx_stag) AXREF_RW(dBy_stag) AXREF_RW(dBz_stag)

#define DECLARE_CCTK_ARGUMENTSX_AsterX_ComputedBFromdBstag                     \
  AXREF_COMMON AXREF_RO(dBx_stag) AXREF_RO(dBy_stag) AXREF_RO(dBz_stag)        \
  AXREF_RW(dBx) AXREF_RW(dBy) AXREF_RW(dBz)

#define DECLARE_CCTK_ARGUMENTSX_AsterX_ComputeBFromdB                          \
  AXREF_COMMON AXREF_METRIC_RO AXREF_RO(dBx) AXREF_RO(dBy) AXREF_RO(dBz)       \
  AXREF_RW(Bvecx) AXREF_RW(Bvecy) AXREF_RW(Bvecz)

#define DECLARE_CCTK_ARGUMENTSX_AsterX_Con2Prim                                \
  AXREF_COMMON AXREF_METRIC_RO AXREF_RO(aster_mask_vc)                         \
  AXREF_RO(Avec_x) AXREF_RO(Avec_y) AXREF_RO(Avec_z)                           \
  AXREF_RW(con2prim_flag) AXREF_RW(aster_mask_cc) AXREF_RW(rho)                \
  AXREF_RW(velx) AXREF_RW(vely) AXREF_RW(velz) AXREF_RW(eps) AXREF_RW(press)   \
  AXREF_RW(Bvecx) AXREF_RW(Bvecy) AXREF_RW(Bvecz) AXREF_RW(temperature)        \
  AXREF_RW(entropy) AXREF_RW(Ye) AXREF_RW(saved_rho) AXREF_RW(saved_velx)      \
  AXREF_RW(saved_vely) AXREF_RW(saved_velz) AXREF_RW(saved_eps)                \
  AXREF_RW(saved_Ye) AXREF_RW(zvec_x) AXREF_RW(zvec_y) AXREF_RW(zvec_z)        \
  AXREF_RW(svec_x) AXREF_RW(svec_y) AXREF_RW(svec_z) AXREF_RW(dens)            \
  AXREF_RW(tau) AXREF_RW(DEnt) AXREF_RW(momx) AXREF_RW(momy) AXREF_RW(momz)    \
  AXREF_RW(DYe) AXREF_RW(dBx) AXREF_RW(dBy) AXREF_RW(dBz)
#define DECLARE_CCTK_ARGUMENTS_AsterX_Con2Prim DECLARE_CCTK_ARGUMENTSX_AsterX_Con2Prim

#define DECLARE_CCTK_ARGUMENTSX_AsterX_Con2Prim_Interpolate_Failed             \
  AXREF_COMMON AXREF_METRIC_RO AXREF_RW(con2prim_flag) AXREF_RW(rho)           \
  AXREF_RW(velx) AXREF_RW(vely) AXREF_RW(velz) AXREF_RW(eps) AXREF_RW(press)   \
  AXREF_RW(saved_rho) AXREF_RW(saved_velx) AXREF_RW(saved_vely)                \
  AXREF_RW(saved_velz) AXREF_RW(saved_eps) AXREF_RW(dens) AXREF_RW(tau)        \
  AXREF_RW(momx) AXREF_RW(momy) AXREF_RW(momz)

#endif
