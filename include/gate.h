/*
 * gate.h - the 18 gate calls (reference include/gate.h:28-73, same signatures).
 *
 * Each call validates its arguments (message "orkan: gate: ..." and exit(1) on a
 * bad qubit or null state, as reference src/gate/gate.c:19-24) and launches one
 * CUDA kernel on the library stream.  PURE applies U to the amplitude vector;
 * MIXED_PACKED / MIXED_TILED apply rho -> U rho U^dagger in place.
 */
#ifndef GATE_H
#define GATE_H

#include "state.h"

#ifdef __cplusplus
extern "C" {
#endif

void x(state_t* state, const qubit_t target);
void y(state_t* state, const qubit_t target);
void z(state_t* state, const qubit_t target);

void h(state_t* state, const qubit_t target);
void s(state_t* state, const qubit_t target);
void sdg(state_t* state, const qubit_t target);
void t(state_t* state, const qubit_t target);
void tdg(state_t* state, const qubit_t target);
void hy(state_t* state, const qubit_t target);

void rx(state_t* state, const qubit_t target, const double theta);
void ry(state_t* state, const qubit_t target, const double theta);
void rz(state_t* state, const qubit_t target, const double theta);
void p(state_t* state, const qubit_t target, const double theta);

void cx(state_t* state, const qubit_t control, const qubit_t target);
void cy(state_t* state, const qubit_t control, const qubit_t target);
void cz(state_t* state, const qubit_t control, const qubit_t target);
void swap_gate(state_t* state, const qubit_t q1, const qubit_t q2);

void ccx(state_t* state, const qubit_t ctrl1, const qubit_t ctrl2, const qubit_t target);

#ifdef __cplusplus
}
#endif

#endif /* GATE_H */
