/*
 * meas.h - diagonal observables (reference include/meas.h:38,57).
 *
 * obs may be a host pointer (copied to the device for the call) or a device
 * pointer (read in place).  Both calls synchronise the library stream and return
 * the value on the host.  The reduction order is fixed, so repeated calls on the
 * same data return bit-identical results.
 */
#ifndef MEAS_H
#define MEAS_H

#include "state.h"

#ifdef __cplusplus
extern "C" {
#endif

/* sum_x obs[x] |psi_x|^2 (PURE) or sum_x obs[x] Re rho_xx (mixed layouts). */
double mean(const state_t *state, const double *obs);

/* sum_x obs[x] conj(bra_x) ket_x; PURE states only (exits otherwise). */
cplx_t matel_diag(const state_t *bra, const state_t *ket, const double *obs);

#ifdef __cplusplus
}
#endif

#endif /* MEAS_H */
