/*
 * internal.h - helpers shared by the host C modules (not installed).
 */
#ifndef ORKAN_HOST_INTERNAL_H
#define ORKAN_HOST_INTERNAL_H

#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>

#include "q_types.h"
#include "state.h"
#include "orkan_cu.h"
#include "orkan_dev.h"

/* Fail-fast validation: "orkan: <module>: <msg>" on stderr, exit(EXIT_FAILURE)
 * (reference src/gate/gate.c:19-24, channel.c:8-13, meas.c:23-28, circ.c:22-27). */
#define ORKAN_VALIDATE(module, cond, msg) do {                  \
    if (!(cond)) {                                              \
        fprintf(stderr, "orkan: %s: %s\n", (module), (msg));    \
        exit(EXIT_FAILURE);                                     \
    }                                                           \
} while (0)

/* A nonzero status from the kernel layer is fatal in the same way. */
void orkan_check_cu(const char *module, const char *what, int rc);

/* Library stream (cudaStream_t as void*). */
void *orkan_stream(void);

/* Device view of a caller array of n doubles: a device pointer is returned as is, a
 * host pointer is copied into the library's staging buffer. */
const double *orkan_device_doubles(const char *module, const double *p, size_t n);

/* Statevector gate queue (fuse.c): enqueue a gate on a PURE state (launched with the
 * next flush, or at once when fusion is off); drop the queue of a state being freed. */
void orkan_pure_gate(state_t *state, const orkan_fgate_t *g, const char *name);
void orkan_fuse_drop(const void *data);

/* Device allocation of len zeroed elements (NULL on failure or injected failure). */
cplx_t *orkan_alloc_state(idx_t len);
void orkan_free_device(void *p);

/* Storage maps (reference src/internal/index.h:57-88). */
static inline idx_t orkan_pack_idx(idx_t dim, idx_t r, idx_t c) {
    return c * (2 * dim - c + 1) / 2 + (r - c);
}
static inline idx_t orkan_tiled_idx(idx_t r, idx_t c) {
    const idx_t tr = r >> LOG_TILE_DIM, tc = c >> LOG_TILE_DIM;
    const idx_t lr = r & (TILE_DIM - 1), lc = c & (TILE_DIM - 1);
    return (tr * (tr + 1) / 2 + tc) * TILE_SIZE + lr * TILE_DIM + lc;
}

#endif /* ORKAN_HOST_INTERNAL_H */
