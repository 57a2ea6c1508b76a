/*
 * circ.c - exp_diag (reference src/circ/circ.c:22-64): validation, the t == 0 early
 * return, and one device pass through orkan_cu_exp_diag.
 */
#include "internal.h"

#include "circ.h"

#define CIRC_VALIDATE(cond, msg) ORKAN_VALIDATE("circ", cond, msg)

static void exp_diag_layout(state_t *state, const double *diag, double t) {
    orkan_flush();
    const size_t dim = (size_t)1 << state->qubits;
    const double *ddiag = orkan_device_doubles("circ", diag, dim);
    orkan_check_cu("circ", "exp_diag",
                   orkan_cu_exp_diag((int)state->type, LOG_TILE_DIM, state->data, state->qubits, ddiag, t,
                                     orkan_stream()));
}

void exp_diag_pure(state_t *state, const double *diag, double t)   { exp_diag_layout(state, diag, t); }
void exp_diag_packed(state_t *state, const double *diag, double t) { exp_diag_layout(state, diag, t); }
void exp_diag_tiled(state_t *state, const double *diag, double t)  { exp_diag_layout(state, diag, t); }

void exp_diag(state_t *state, const double *diag, double t) {
    CIRC_VALIDATE(state && state->data, "exp_diag: null state or data pointer");
    CIRC_VALIDATE(diag, "exp_diag: null diagonal pointer");
    if (t == 0.0) return;
    switch (state->type) {
        case PURE:         exp_diag_pure(state, diag, t); break;
        case MIXED_PACKED: exp_diag_packed(state, diag, t); break;
        case MIXED_TILED:  exp_diag_tiled(state, diag, t); break;
        default:           CIRC_VALIDATE(0, "exp_diag: invalid state type");
    }
}
