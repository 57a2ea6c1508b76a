/*
 * state.c - state lifecycle on device storage (reference src/state/state.c,
 * state_pure.c, state_packed.c, state_tiled.c).
 *
 * Storage is cudaMalloc'd (256-byte aligned, zero-filled on the library stream).
 * Ownership follows the reference (state.c:60-108): state_init frees previous data,
 * takes ownership of a caller buffer and nulls the caller's pointer; state_free is
 * idempotent; allocation failure leaves data == NULL and qubits == 0 with a message.
 */
#include "internal.h"

#include <cuda_runtime_api.h>
#include <math.h>
#include <string.h>

/* ---- storage lengths (reference state_pure.c:25-28, state_packed.c:36-54,
 *      state_tiled.c:68-81) ---------------------------------------------------- */
idx_t state_pure_len(qubit_t qubits) { return POW2(qubits, idx_t); }

idx_t state_packed_len(qubit_t qubits) {
    const idx_t dim = POW2(qubits, idx_t);
    return qubits == 0 ? 1 : (dim >> 1) * (dim + 1);
}

idx_t state_tiled_len(qubit_t qubits) {
    const idx_t dim = POW2(qubits, idx_t);
    const idx_t nt = (dim + TILE_DIM - 1) >> LOG_TILE_DIM;
    return (nt * (nt + 1) >> 1) * TILE_SIZE;
}

idx_t state_len(const state_t *state) {
    ORKAN_VALIDATE("state", state != NULL, "state_len: null state");
    switch (state->type) {
        case PURE:         return state_pure_len(state->qubits);
        case MIXED_PACKED: return state_packed_len(state->qubits);
        case MIXED_TILED:  return state_tiled_len(state->qubits);
        default:           ORKAN_VALIDATE("state", 0, "state_len: invalid state type");
    }
    return 0;
}

static int layout_code(const state_t *s) { return (int)s->type; }

/* ---- lifecycle -------------------------------------------------------------- */
static int is_device_buffer(const void *p) {
    struct cudaPointerAttributes a;
    memset(&a, 0, sizeof(a));
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeDevice;
}

void state_init(state_t *state, const qubit_t qubits, cplx_t **data) {
    ORKAN_VALIDATE("state", state != NULL, "state_init: null state");
    orkan_flush();
    if (state->data) {
        orkan_free_device(state->data);
        state->data = NULL;
    }
    state->qubits = qubits;
    const idx_t len = state_len(state);

    if (data && *data) {
        if (is_device_buffer(*data)) {
            state->data = *data;                      /* adopt a cudaMalloc'd buffer */
        } else {
            state->data = orkan_alloc_state(len);
            if (!state->data) {
                fprintf(stderr, "state_init(): device allocation failed for %zu elements\n", (size_t)len);
                state->qubits = 0;
                free(*data);
                *data = NULL;
                return;
            }
            cudaError_t e = cudaMemcpyAsync(state->data, *data, (size_t)len * sizeof(cplx_t),
                                            cudaMemcpyHostToDevice, (cudaStream_t)orkan_stream());
            if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)orkan_stream());
            orkan_check_cu("state", "state_init: host-to-device copy", (int)e);
            free(*data);
        }
        *data = NULL;
    } else {
        state->data = orkan_alloc_state(len);
        if (!state->data) {
            fprintf(stderr, "state_init(): device allocation failed for %zu elements\n", (size_t)len);
            state->qubits = 0;
        }
    }
}

void state_free(state_t *state) {
    if (!state) return;
    orkan_fuse_drop(state->data);
    orkan_free_device(state->data);
    state->data = NULL;
    state->qubits = 0;
}

void state_plus(state_t *state, const qubit_t qubits) {
    ORKAN_VALIDATE("state", state != NULL, "state_plus: null state");
    state_init(state, qubits, NULL);
    if (!state->data) return;
    const idx_t dim = POW2(qubits, idx_t);
    /* PURE: 1/sqrt(2^n); mixed: every element of |+><+| is 1/2^n */
    const double v = state->type == PURE ? 1.0 / sqrt((double)dim) : 1.0 / (double)dim;
    orkan_check_cu("state", "state_plus",
                   orkan_cu_fill(layout_code(state), LOG_TILE_DIM, state->data, qubits, v, 0.0, orkan_stream()));
}

void state_pure_plus(state_t *state, qubit_t qubits) { state->type = PURE; state_plus(state, qubits); }
void state_packed_plus(state_t *state, qubit_t qubits) { state->type = MIXED_PACKED; state_plus(state, qubits); }
void state_tiled_plus(state_t *state, qubit_t qubits) { state->type = MIXED_TILED; state_plus(state, qubits); }

state_t state_cp(const state_t *state) {
    ORKAN_VALIDATE("state", state != NULL && state->data != NULL, "state_cp: null state or data");
    orkan_flush();
    state_t out = *state;
    const idx_t len = state_len(state);
    out.data = orkan_alloc_state(len);
    if (!out.data) {
        fprintf(stderr, "state_cp(): allocation failed\n");
        out.qubits = 0;
        return out;
    }
    cudaError_t e = cudaMemcpyAsync(out.data, state->data, (size_t)len * sizeof(cplx_t), cudaMemcpyDeviceToDevice,
                                    (cudaStream_t)orkan_stream());
    orkan_check_cu("state", "state_cp: device-to-device copy", (int)e);
    return out;
}

/* ---- element access (reference state_pure.c:46-56, state_packed.c:79-104,
 *      state_tiled.c:117-150) --------------------------------------------------- */
static cplx_t read_elem(const state_t *s, idx_t i) {
    orkan_flush();
    cplx_t v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, s->data + i, sizeof(cplx_t), cudaMemcpyDeviceToHost,
                                    (cudaStream_t)orkan_stream());
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)orkan_stream());
    orkan_check_cu("state", "state_get: device-to-host copy", (int)e);
    return v;
}

static void write_elem(state_t *s, idx_t i, cplx_t v) {
    orkan_flush();
    cudaError_t e = cudaMemcpyAsync(s->data + i, &v, sizeof(cplx_t), cudaMemcpyHostToDevice,
                                    (cudaStream_t)orkan_stream());
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)orkan_stream());
    orkan_check_cu("state", "state_set: host-to-device copy", (int)e);
}

cplx_t state_pure_get(const state_t *state, idx_t row) { return read_elem(state, row); }
void state_pure_set(state_t *state, idx_t row, cplx_t val) { write_elem(state, row, val); }

cplx_t state_packed_get(const state_t *state, idx_t row, idx_t col) {
    const idx_t dim = POW2(state->qubits, idx_t);
    return row >= col ? read_elem(state, orkan_pack_idx(dim, row, col))
                      : conj(read_elem(state, orkan_pack_idx(dim, col, row)));
}

void state_packed_set(state_t *state, idx_t row, idx_t col, cplx_t val) {
    const idx_t dim = POW2(state->qubits, idx_t);
    if (row >= col) write_elem(state, orkan_pack_idx(dim, row, col), val);
    else            write_elem(state, orkan_pack_idx(dim, col, row), conj(val));
}

cplx_t state_tiled_get(const state_t *state, idx_t row, idx_t col) {
    return row >= col ? read_elem(state, orkan_tiled_idx(row, col))
                      : conj(read_elem(state, orkan_tiled_idx(col, row)));
}

void state_tiled_set(state_t *state, idx_t row, idx_t col, cplx_t val) {
    const int same_tile = (row >> LOG_TILE_DIM) == (col >> LOG_TILE_DIM);
    if (row >= col) {
        write_elem(state, orkan_tiled_idx(row, col), val);
        if (same_tile && row != col) write_elem(state, orkan_tiled_idx(col, row), conj(val));
    } else {
        write_elem(state, orkan_tiled_idx(col, row), conj(val));
        if (same_tile) write_elem(state, orkan_tiled_idx(row, col), val);
    }
}

cplx_t state_get(const state_t *state, idx_t row, idx_t col) {
    ORKAN_VALIDATE("state", state != NULL && state->data != NULL, "state_get: null state or data");
    const idx_t dim = POW2(state->qubits, idx_t);
    switch (state->type) {
        case PURE:
            ORKAN_VALIDATE("state", row < dim && col == 0, "state_get: index out of range");
            return state_pure_get(state, row);
        case MIXED_PACKED:
            ORKAN_VALIDATE("state", row < dim && col < dim, "state_get: index out of range");
            return state_packed_get(state, row, col);
        case MIXED_TILED:
            ORKAN_VALIDATE("state", row < dim && col < dim, "state_get: index out of range");
            return state_tiled_get(state, row, col);
        default:
            ORKAN_VALIDATE("state", 0, "state_get: invalid state type");
    }
    return 0;
}

void state_set(state_t *state, idx_t row, idx_t col, cplx_t val) {
    ORKAN_VALIDATE("state", state != NULL && state->data != NULL, "state_set: null state or data");
    const idx_t dim = POW2(state->qubits, idx_t);
    switch (state->type) {
        case PURE:
            ORKAN_VALIDATE("state", row < dim && col == 0, "state_set: index out of range");
            state_pure_set(state, row, val);
            break;
        case MIXED_PACKED:
            ORKAN_VALIDATE("state", row < dim && col < dim, "state_set: index out of range");
            state_packed_set(state, row, col, val);
            break;
        case MIXED_TILED:
            ORKAN_VALIDATE("state", row < dim && col < dim, "state_set: index out of range");
            state_tiled_set(state, row, col, val);
            break;
        default:
            ORKAN_VALIDATE("state", 0, "state_set: invalid state type");
    }
}

/* ---- printing: copy to the host, then print with 7 decimals like the reference -- */
static void print_c(cplx_t v) {
    printf("%.7f", creal(v));
    if (cimag(v) >= 0) printf("+i%.7f", cimag(v));
    else               printf("-i%.7f", -cimag(v));
}

static cplx_t *download_all(const state_t *s) {
    const idx_t len = state_len(s);
    cplx_t *h = (cplx_t *)malloc((size_t)len * sizeof(cplx_t));
    ORKAN_VALIDATE("state", h != NULL, "state_print: host allocation failed");
    orkan_check_cu("state", "state_print: download", orkan_state_download(s, h));
    return h;
}

static void print_matrix(const state_t *s, const cplx_t *h) {
    const idx_t dim = POW2(s->qubits, idx_t);
    for (idx_t r = 0; r < dim; ++r) {
        printf("[");
        for (idx_t c = 0; c < dim; ++c) {
            cplx_t v;
            if (s->type == MIXED_PACKED) v = r >= c ? h[orkan_pack_idx(dim, r, c)] : conj(h[orkan_pack_idx(dim, c, r)]);
            else                         v = r >= c ? h[orkan_tiled_idx(r, c)] : conj(h[orkan_tiled_idx(c, r)]);
            if (c) printf(", ");
            print_c(v);
        }
        printf("]\n");
    }
}

void state_pure_print(const state_t *state) {
    printf("Type: PURE\nQubits: %u\n", state->qubits);
    cplx_t *h = download_all(state);
    const idx_t dim = POW2(state->qubits, idx_t);
    printf("[");
    for (idx_t i = 0; i < dim; ++i) {
        if (i) printf(", ");
        print_c(h[i]);
    }
    printf("]\n");
    free(h);
}

void state_packed_print(const state_t *state) {
    printf("Type: MIXED_PACKED\nQubits: %u\n", state->qubits);
    cplx_t *h = download_all(state);
    print_matrix(state, h);
    free(h);
}

void state_tiled_print(const state_t *state) {
    printf("Type: MIXED_TILED\nQubits: %u\n", state->qubits);
    cplx_t *h = download_all(state);
    print_matrix(state, h);
    free(h);
}

void state_print(const state_t *state) {
    ORKAN_VALIDATE("state", state != NULL && state->data != NULL, "state_print: null state or data");
    switch (state->type) {
        case PURE:         state_pure_print(state); break;
        case MIXED_PACKED: state_packed_print(state); break;
        case MIXED_TILED:  state_tiled_print(state); break;
        default:           ORKAN_VALIDATE("state", 0, "state_print: invalid state type");
    }
}
