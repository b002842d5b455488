/*
 * axo.h -- the oracle restatement (test infrastructure only).
 *
 * A plain, single-threaded-per-point C++ restatement of the reference's hot
 * path, used only by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline to check the engine.  It exports the same `ora_*` C ABI as the
 * reference harness in oracle/refshim/axref_harness.cpp, so a test can run
 * the restatement and the reference's own sources on identical inputs and
 * demand bit-equality (both are compiled with -ffp-contract=off).  Nothing in
 * the product library links or includes it.
 */
#ifndef AXO_H
#define AXO_H

#include "../include/asterx_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

const char *ora_last_error(void);
int ora_bind(const char *name, double *ptr);
int ora_setup(const axb_box *box, const axb_params *params, int iteration);
void ora_set_ext(int ext_c, int ext_v);
int ora_eos_idealgas(double gamma, double umass, double rho_min, double rho_max,
                     double eps_min, double eps_max, double ye_min, double ye_max,
                     double poly_gamma, double poly_k);
int ora_eos_tabulated(int nrho, int ntemp, int nye, const double *logrho,
                      const double *logtemp, const double *yes,
                      const double *table, double energy_shift,
                      double poly_gamma, double poly_k);
void ora_eos_tab_ranges(double *out8);
int ora_fluxes(void);
int ora_sources(void);
int ora_rhs(void);
int ora_bstag(void);
int ora_dB(void);
int ora_c2p(void);
void ora_reconstruct(int method, const double *v, const double *press,
                     const double *vel, int is_rho, int is_press, double *out);
void ora_eigen(const double *in, double *lam);
double ora_riemann(int flux_type, const double *lam, double uL, double uR,
                   double fL, double fR);
void ora_prim2con(const double *g6, const double *prim, double *cons);
int ora_c2p_point(int solver, double *cons, const double *g6, const double *seed,
                  const double *atmo, double *prim, int *rep3);
double ora_eos_tab_query(int which, double rho, double x, double ye,
                         double *eps_io);

#ifdef __cplusplus
}
#endif

#endif
