/*
 * state.h - quantum state handle and its lifecycle (device-resident storage).
 *
 * Same types and signatures as the reference include/state.h:31-143.  The one
 * semantic difference of this build: state_t.data points to GPU memory.  Host
 * code must not dereference it; use state_get/state_set for single elements and
 * orkan_state_download/orkan_state_upload (orkan_dev.h) for bulk copies.
 *
 * Storage layouts (identical element order to the reference):
 *   PURE          2^n amplitudes, index = basis state.
 *   MIXED_PACKED  lower triangle, column-major: (r,c), r>=c at c*(2d-c+1)/2 + (r-c).
 *   MIXED_TILED   lower-triangular grid of TILE_DIM x TILE_DIM tiles, tiles in
 *                 row-major tile order (tr*(tr+1)/2 + tc), elements row-major in a
 *                 tile; diagonal tiles hold both triangles (upper = conj(lower));
 *                 for 2^n < TILE_DIM a single tile whose dim x dim corner is live.
 */
#ifndef STATE_H
#define STATE_H

#include "q_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum state_type {
    PURE,
    MIXED_PACKED,
    MIXED_TILED
} state_type_t;

typedef struct state {
    state_type_t type;
    cplx_t *data;       /* device pointer in this build */
    qubit_t qubits;
} state_t;

typedef void (*qop_t)(state_t *state);

/* Number of complex elements of the storage (reference src/state/state.c:43-58). */
idx_t state_len(const state_t *state);

/* Allocate zeroed device storage, or take ownership of *data (reference
 * state.c:60-99).  A host buffer from malloc() is copied to the device, freed and
 * *data set to NULL; a device buffer from cudaMalloc() is adopted as is. */
void state_init(state_t *state, qubit_t qubits, cplx_t **data);

/* Release the storage; safe to call twice (reference state.c:102-108). */
void state_free(state_t *state);

/* |+>^n: PURE amplitudes 2^(-n/2); mixed layouts every stored element 1/2^n
 * (reference state_pure.c:30-43, state_packed.c:57-76, state_tiled.c:84-114). */
void state_plus(state_t *state, qubit_t qubits);

/* Deep device-to-device copy; data == NULL on allocation failure (state.c:130-148). */
state_t state_cp(const state_t *state);

/* Print type, qubits and elements (copies the storage to the host first). */
void state_print(const state_t *state);

/* Element access with Hermitian mapping for mixed states (state.c:170-204). */
cplx_t state_get(const state_t *state, idx_t row, idx_t col);
void state_set(state_t *state, idx_t row, idx_t col, cplx_t val);

#ifdef __cplusplus
}
#endif

#endif /* STATE_H */
