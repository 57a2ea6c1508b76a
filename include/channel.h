/*
 * channel.h - Kraus and superoperator channels (reference include/channel.h:28-67).
 *
 * kraus_t / superop_t hold HOST matrices (row-major), exactly as in the reference.
 * kraus_to_superop runs on the host and returns calloc'd data the caller frees.
 * channel_1q copies the 16 superoperator entries into the kernel's parameters and
 * updates the device-resident density matrix in one pass.
 */
#ifndef CHANNEL_H
#define CHANNEL_H

#include "state.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  qubit_t n_qubits;
  uint64_t n_terms;
  cplx_t* data;
} kraus_t;

typedef struct {
  qubit_t n_qubits;
  cplx_t* data;
} superop_t;

/* S[(i,j),(k,l)] = sum_a K_a[i,k] * conj(K_a[j,l]), row-major (N^2 x N^2). */
superop_t kraus_to_superop(const kraus_t *kraus);

/* vec(rho_2x2)' = S vec(rho_2x2) on every 2x2 block of the target qubit;
 * vec order (00, 01, 10, 11).  Mixed states only; exits on PURE. */
void channel_1q(state_t *state, const superop_t *sop, qubit_t target);

#ifdef __cplusplus
}
#endif

#endif /* CHANNEL_H */
