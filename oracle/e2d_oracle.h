/*
 * e2d_oracle.h — CPU restatement of the CFFC reference's Euler2D residual,
 * explicit multistage time marching and residual norms, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU library is compared
 * against: only tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py load it.  The product (libcffc_e2d.so) neither links nor calls it.
 *
 * The restatement follows the reference routine by routine and keeps its
 * floating-point operation order, so that with FMA contraction off it
 * reproduces the compiled reference bit for bit; it is pinned against the
 * reference itself (oracle/_ref/e2d_ref_harness, oracle/Makefile) by the
 * golden vectors in tests/golden/ (tests/golden/make_golden.py).
 *
 * The API mirrors include/cffc_e2d.h so one test can drive either.
 */
#ifndef E2D_ORACLE_H
#define E2D_ORACLE_H
#include "../include/cffc_e2d.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct e2d_oracle e2d_oracle;

e2d_oracle *e2d_oracle_create(const e2d_blocks_desc *desc, const e2d_scheme *scheme, int *err);
void e2d_oracle_destroy(e2d_oracle *o);
int e2d_oracle_set_state(e2d_oracle *o, const double *W);
int e2d_oracle_get_state(e2d_oracle *o, double *W, double *U);
int e2d_oracle_fill_ghosts(e2d_oracle *o);
int e2d_oracle_residual(e2d_oracle *o, double *dUdt);
int e2d_oracle_get_reconstruction(e2d_oracle *o, double *dWdx, double *dWdy, double *phi);
int e2d_oracle_rk_steps(e2d_oracle *o, int n_steps, double *hist);
int e2d_oracle_geometry(e2d_oracle *o, double *xc, double *yc, double *area);

#ifdef __cplusplus
}
#endif
#endif
