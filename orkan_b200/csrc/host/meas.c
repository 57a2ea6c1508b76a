/*
 * meas.c - mean and matel_diag (reference src/meas/meas.c:23-74): validation in C,
 * deterministic device reductions through orkan_cu_mean / orkan_cu_matel_diag.
 */
#include "internal.h"

#include "meas.h"

#define MEAS_VALIDATE(cond, msg) ORKAN_VALIDATE("meas", cond, msg)

static double mean_layout(const state_t *state, const double *obs) {
    orkan_flush();
    const size_t dim = (size_t)1 << state->qubits;
    const double *dobs = orkan_device_doubles("meas", obs, dim);
    double r = 0.0;
    orkan_check_cu("meas", "mean",
                   orkan_cu_mean((int)state->type, LOG_TILE_DIM, state->data, state->qubits, dobs, &r, orkan_stream()));
    return r;
}

double mean_pure(const state_t *state, const double *obs)   { return mean_layout(state, obs); }
double mean_packed(const state_t *state, const double *obs) { return mean_layout(state, obs); }
double mean_tiled(const state_t *state, const double *obs)  { return mean_layout(state, obs); }

cplx_t matel_diag_pure(const state_t *bra, const state_t *ket, const double *obs) {
    orkan_flush();
    const size_t dim = (size_t)1 << bra->qubits;
    const double *dobs = orkan_device_doubles("meas", obs, dim);
    double r[2] = {0.0, 0.0};
    orkan_check_cu("meas", "matel_diag",
                   orkan_cu_matel_diag(bra->data, ket->data, bra->qubits, dobs, r, orkan_stream()));
    return r[0] + r[1] * I;
}

double mean(const state_t *state, const double *obs) {
    MEAS_VALIDATE(state && state->data, "mean: null state or data pointer");
    MEAS_VALIDATE(obs, "mean: null observable pointer");
    switch (state->type) {
        case PURE:         return mean_pure(state, obs);
        case MIXED_PACKED: return mean_packed(state, obs);
        case MIXED_TILED:  return mean_tiled(state, obs);
        default:           MEAS_VALIDATE(0, "mean: invalid state type");
    }
    return 0.0;
}

cplx_t matel_diag(const state_t *bra, const state_t *ket, const double *obs) {
    MEAS_VALIDATE(bra && bra->data, "matel_diag: null bra state or data pointer");
    MEAS_VALIDATE(ket && ket->data, "matel_diag: null ket state or data pointer");
    MEAS_VALIDATE(obs, "matel_diag: null observable pointer");
    MEAS_VALIDATE(bra->qubits == ket->qubits, "matel_diag: qubit count mismatch");
    MEAS_VALIDATE(bra->type == PURE, "matel_diag: bra must be PURE (mixed not supported)");
    MEAS_VALIDATE(ket->type == PURE, "matel_diag: ket must be PURE (mixed not supported)");
    return matel_diag_pure(bra, ket, obs);
}
