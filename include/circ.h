/*
 * circ.h - diagonal evolution (reference include/circ.h:41).
 *
 * exp_diag(state, diag, t):  PURE   psi_x    *= exp(-i diag[x] t)
 *                            mixed  rho_rc   *= exp(-i (diag[r] - diag[c]) t)
 * No implicit factor 1/2.  t == 0 returns without touching the state.  diag may be
 * a host pointer (copied for the call) or a device pointer.
 */
#ifndef CIRC_H
#define CIRC_H

#include "state.h"

#ifdef __cplusplus
extern "C" {
#endif

void exp_diag(state_t *state, const double *diag, double t);

#ifdef __cplusplus
}
#endif

#endif /* CIRC_H */
