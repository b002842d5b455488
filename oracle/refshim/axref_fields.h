// Test infrastructure only: every grid function the reference hot path
// touches, as one X-macro list.  The harness binds a host array to each name;
// the argument macros in cctk_Arguments.h turn the names into GF3D2 views.
#ifndef AXREF_FIELDS_H
#define AXREF_FIELDS_H

#define AXREF_FIELD_LIST(X)                                                    \
  X(gxx) X(gxy) X(gxz) X(gyy) X(gyz) X(gzz) X(alp) X(betax) X(betay) X(betaz)  \
  X(kxx) X(kxy) X(kxz) X(kyy) X(kyz) X(kzz)                                    \
  X(rho) X(velx) X(vely) X(velz) X(eps) X(press) X(temperature) X(Ye)          \
  X(entropy) X(Bvecx) X(Bvecy) X(Bvecz)                                        \
  X(dens) X(momx) X(momy) X(momz) X(tau) X(DYe) X(DEnt)                        \
  X(densrhs) X(momxrhs) X(momyrhs) X(momzrhs) X(taurhs) X(DYe_rhs) X(DEntrhs)  \
  X(fxdens) X(fxmomx) X(fxmomy) X(fxmomz) X(fxtau) X(fxDYe) X(fxDEnt)          \
  X(fxBx) X(fxBy) X(fxBz)                                                      \
  X(fydens) X(fymomx) X(fymomy) X(fymomz) X(fytau) X(fyDYe) X(fyDEnt)          \
  X(fyBx) X(fyBy) X(fyBz)                                                      \
  X(fzdens) X(fzmomx) X(fzmomy) X(fzmomz) X(fztau) X(fzDYe) X(fzDEnt)          \
  X(fzBx) X(fzBy) X(fzBz)                                                      \
  X(Avec_x) X(Avec_y) X(Avec_z) X(Psi)                                         \
  X(Avec_x_rhs) X(Avec_y_rhs) X(Avec_z_rhs) X(Psi_rhs)                         \
  X(Fx) X(Fy) X(Fz) X(Fbetax) X(Fbetay) X(Fbetaz) X(G)                         \
  X(dBx_stag) X(dBy_stag) X(dBz_stag) X(dBx) X(dBy) X(dBz)                     \
  X(con2prim_flag) X(saved_rho) X(saved_velx) X(saved_vely) X(saved_velz)      \
  X(saved_eps) X(saved_Ye)                                                     \
  X(zvec_x) X(zvec_y) X(zvec_z) X(svec_x) X(svec_y) X(svec_z)                  \
  X(vtilde_y_xface) X(vtilde_z_xface) X(vtilde_x_yface) X(vtilde_z_yface)      \
  X(vtilde_x_zface) X(vtilde_y_zface)                                          \
  X(amax_xface) X(amin_xface) X(amax_yface) X(amin_yface) X(amax_zface)        \
  X(amin_zface) X(aster_mask_vc) X(aster_mask_cc)                             \
  X(eTtt) X(eTtx) X(eTty) X(eTtz) X(eTxx) X(eTxy) X(eTxz) X(eTyy) X(eTyz)      \
  X(eTzz) X(regrid_error)

enum axref_field_id {
#define AXREF_ENUM(name) AXREF_F_##name,
  AXREF_FIELD_LIST(AXREF_ENUM)
#undef AXREF_ENUM
  AXREF_NFIELDS
};

#endif
