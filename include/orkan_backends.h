/*
 * orkan_backends.h - per-layout backend entry points.
 *
 * The reference liborkan.so exports these names besides the public API, and its test
 * and profiling harnesses call them directly (e.g. x_tiled, h_packed, channel_tiled_1q,
 * mean_tiled, single_from_mat; reference docs/PROFILE.md:66 and
 * test/gate/test_gate_tiled_1q.c).  This library exports the same names with the same
 * signatures; each launches the device kernel for its layout.  They perform no argument
 * validation (the public dispatchers do), exactly as in the reference.
 */
#ifndef ORKAN_BACKENDS_H
#define ORKAN_BACKENDS_H

#include "state.h"

#ifdef __cplusplus
extern "C" {
#endif

/* state (reference src/state/state_internal.h:22-52) */
idx_t  state_pure_len(qubit_t qubits);
void   state_pure_plus(state_t *state, qubit_t qubits);
cplx_t state_pure_get(const state_t *state, idx_t row);
void   state_pure_set(state_t *state, idx_t row, cplx_t val);
void   state_pure_print(const state_t *state);
idx_t  state_packed_len(qubit_t qubits);
void   state_packed_plus(state_t *state, qubit_t qubits);
cplx_t state_packed_get(const state_t *state, idx_t row, idx_t col);
void   state_packed_set(state_t *state, idx_t row, idx_t col, cplx_t val);
void   state_packed_print(const state_t *state);
idx_t  state_tiled_len(qubit_t qubits);
void   state_tiled_plus(state_t *state, qubit_t qubits);
cplx_t state_tiled_get(const state_t *state, idx_t row, idx_t col);
void   state_tiled_set(state_t *state, idx_t row, idx_t col, cplx_t val);
void   state_tiled_print(const state_t *state);

/* gates (reference src/gate/gate.c:35-112) */
#define ORKAN_DECLARE_GATE_BACKENDS(L)                                              \
    void x_##L(state_t *state, qubit_t target);                                     \
    void y_##L(state_t *state, qubit_t target);                                     \
    void z_##L(state_t *state, qubit_t target);                                     \
    void h_##L(state_t *state, qubit_t target);                                     \
    void s_##L(state_t *state, qubit_t target);                                     \
    void sdg_##L(state_t *state, qubit_t target);                                   \
    void t_##L(state_t *state, qubit_t target);                                     \
    void tdg_##L(state_t *state, qubit_t target);                                   \
    void hy_##L(state_t *state, qubit_t target);                                    \
    void rx_##L(state_t *state, qubit_t target, double theta);                      \
    void ry_##L(state_t *state, qubit_t target, double theta);                      \
    void rz_##L(state_t *state, qubit_t target, double theta);                      \
    void p_##L(state_t *state, qubit_t target, double theta);                       \
    void cx_##L(state_t *state, qubit_t control, qubit_t target);                   \
    void cy_##L(state_t *state, qubit_t control, qubit_t target);                   \
    void cz_##L(state_t *state, qubit_t control, qubit_t target);                   \
    void swap_##L(state_t *state, qubit_t q1, qubit_t q2);                          \
    void ccx_##L(state_t *state, qubit_t ctrl1, qubit_t ctrl2, qubit_t target);
ORKAN_DECLARE_GATE_BACKENDS(pure)
ORKAN_DECLARE_GATE_BACKENDS(packed)
ORKAN_DECLARE_GATE_BACKENDS(tiled)
#undef ORKAN_DECLARE_GATE_BACKENDS

/* generic unitaries on density matrices, mat column-major (reference
 * src/gate/tiled/gate_tiled.h:36, gate_tiled_2q.c:3) */
void single_from_mat(state_t *state, qubit_t target, const cplx_t *mat);
void two_from_mat(state_t *state, qubit_t q1, qubit_t q2, const cplx_t *mat);

/* channels (reference src/channel/channel.c:58-59) */
void channel_packed_1q(state_t *state, const cplx_t *sop, qubit_t target);
void channel_tiled_1q(state_t *state, const cplx_t *sop, qubit_t target);

/* measurement (reference src/meas/meas.c:36-40) */
double mean_pure(const state_t *state, const double *obs);
double mean_packed(const state_t *state, const double *obs);
double mean_tiled(const state_t *state, const double *obs);
cplx_t matel_diag_pure(const state_t *bra, const state_t *ket, const double *obs);

/* circuit (reference src/circ/circ.c:36-38) */
void exp_diag_pure(state_t *state, const double *diag, double t);
void exp_diag_packed(state_t *state, const double *diag, double t);
void exp_diag_tiled(state_t *state, const double *diag, double t);

#ifdef __cplusplus
}
#endif

#endif /* ORKAN_BACKENDS_H */
