/* ============================================================================
 *  lbm_oracle.h -- TEST INFRASTRUCTURE ONLY: plain-C restatement of the
 *  reference solver's hot path, used as the checker of the CUDA library.
 *  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 *  load it. It is never part of the product path.
 *
 *  Pinned against the reference itself: tests/test_oracle.py compares it
 *  bit-for-bit with the reference compiled from its own sources
 *  (oracle/_ref/libref_harness.so) and with the reference's shipped outputs.
 * ==========================================================================*/
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include "../include/lbmgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lbo_state lbo_state;

lbo_state* lbo_create(const lbmgpu_params* p);
void lbo_destroy(lbo_state* s);
void lbo_step(lbo_state* s);
void lbo_advance_squirmer(lbo_state* s);
void lbo_correct_mass(lbo_state* s);
int  lbo_run(lbo_state* s, int nsteps, double* traj, int max_rows);
long lbo_ncells(const lbo_state* s);
long lbo_time(const lbo_state* s);
void lbo_get_f(const lbo_state* s, double* out);
void lbo_set_f(lbo_state* s, const double* in);
void lbo_get_fields(const lbo_state* s, unsigned char* flag, double* rho, double* u3);
void lbo_set_flags(lbo_state* s, const unsigned char* flag);
void lbo_squirmer_state(const lbo_state* s, double* o);
void lbo_set_squirmer_state(lbo_state* s, const double* X, const double* e, const double* U, const double* W);
void lbo_wall_force(const lbo_state* s, double* o);
void lbo_diag(const lbo_state* s, double* o);
double lbo_duct_velocity(double y, double z, double a, double b, double G, double mu);
double lbo_poiseuille_error(const lbo_state* s);

#ifdef __cplusplus
}
#endif
#endif
