/*
 * bench_orkan_b200.c - B200 backends for the reference's gate benchmark CLI
 * (benchmark/include/bench.h:78-96: the bench_backend_t vtable; benchmark/src/bench_orkan.c
 * is the CPU version these mirror).
 *
 * This file is compiled inside the reference's benchmark (it includes its bench.h) and
 * linked against liborkan_b200.so.  The library keeps the reference's public API, so the
 * gate calls are the same as in bench_orkan.c; two things differ because state storage
 * lives in device memory:
 *   - init fills the Hermitian start state in a host buffer with the benchmark's own
 *     bench_init_hermitian_{tiled,packed} and uploads it (orkan_state_upload), instead of
 *     writing through state->data;
 *   - apply waits for the gate to finish (orkan_sync) before returning, so that the
 *     harness's host clock around a sequence of applies measures completed gates.
 * touch_bytes are the reference's formulas (2 x storage bytes).  available() checks that
 * the storage fits in the device's free memory.
 *
 * The Kraus benchmark's vtable (benchmark/include/bench_kraus.h:54-62; the CPU version is
 * benchmark/src/bench_kraus_orkan.c) is implemented here too when BENCH_B200_KRAUS is
 * defined: the superoperator is built once at init with kraus_to_superop (not timed) and
 * apply calls channel_1q.  With BENCH_B200_AS_REFERENCE the vtables are also exported under
 * the reference's own names (orkan_tiled_backend, orkan_packed_backend and the
 * kraus_orkan_* pair), so the reference's unmodified bench_main.c / bench_kraus_main.c,
 * linked with this file instead of bench_orkan.c / bench_kraus_orkan.c, run their
 * "orkan" rows on the B200.
 */
#ifdef BENCH_B200_KRAUS
#include "bench_kraus.h"
#else
#include "bench.h"
#endif

#include <cuda_runtime.h>

#include "orkan_dev.h"

typedef void (*b200_apply_fn)(state_t *s, const qubit_t *p, double par);

typedef struct {
    state_t      *state;
    b200_apply_fn apply;
    double        par;
} b200_ctx_t;

static void g_x(state_t *st, const qubit_t *p, double a)   { (void)a; x(st, p[0]); }
static void g_y(state_t *st, const qubit_t *p, double a)   { (void)a; y(st, p[0]); }
static void g_z(state_t *st, const qubit_t *p, double a)   { (void)a; z(st, p[0]); }
static void g_h(state_t *st, const qubit_t *p, double a)   { (void)a; h(st, p[0]); }
static void g_s(state_t *st, const qubit_t *p, double a)   { (void)a; s(st, p[0]); }
static void g_t(state_t *st, const qubit_t *p, double a)   { (void)a; t(st, p[0]); }
static void g_rx(state_t *st, const qubit_t *p, double a)  { rx(st, p[0], a); }
static void g_ry(state_t *st, const qubit_t *p, double a)  { ry(st, p[0], a); }
static void g_rz(state_t *st, const qubit_t *p, double a)  { rz(st, p[0], a); }
static void g_cx(state_t *st, const qubit_t *p, double a)  { (void)a; cx(st, p[0], p[1]); }
static void g_cy(state_t *st, const qubit_t *p, double a)  { (void)a; cy(st, p[0], p[1]); }
static void g_cz(state_t *st, const qubit_t *p, double a)  { (void)a; cz(st, p[0], p[1]); }
static void g_ccx(state_t *st, const qubit_t *p, double a) { (void)a; ccx(st, p[0], p[1], p[2]); }

static b200_apply_fn b200_resolve(bench_gate_id_t gate) {
    switch (gate) {
    case BG_X:   return g_x;
    case BG_Y:   return g_y;
    case BG_Z:   return g_z;
    case BG_H:   return g_h;
    case BG_S:   return g_s;
    case BG_T:   return g_t;
    case BG_RX:  return g_rx;
    case BG_RY:  return g_ry;
    case BG_RZ:  return g_rz;
    case BG_CX:  return g_cx;
    case BG_CY:  return g_cy;
    case BG_CZ:  return g_cz;
    case BG_CCX: return g_ccx;
    default:
        fprintf(stderr, "bench_orkan_b200: unknown gate id %d\n", (int)gate);
        abort();
    }
}

static void b200_apply(void *ctx, const qubit_t *pos) {
    b200_ctx_t *c = (b200_ctx_t *)ctx;
    c->apply(c->state, pos, c->par);
    orkan_sync();
}

static void b200_cleanup(void *ctx) {
    b200_ctx_t *c = (b200_ctx_t *)ctx;
    state_free(c->state);
    free(c->state);
    free(c);
}

/* A device state of the given layout holding the benchmark's Hermitian start state. */
static void *b200_init(state_type_t type, qubit_t qubits, bench_gate_id_t gate, double par) {
    b200_ctx_t *c = calloc(1, sizeof(b200_ctx_t));
    if (!c) return NULL;
    c->state = calloc(1, sizeof(state_t));
    if (!c->state) { free(c); return NULL; }
    c->state->type = type;
    state_init(c->state, qubits, NULL);
    if (!c->state->data) { free(c->state); free(c); return NULL; }
    const idx_t len = state_len(c->state);
    cplx_t *host = calloc(len, sizeof(cplx_t));
    if (!host) { b200_cleanup(c); return NULL; }
    if (type == MIXED_TILED) bench_init_hermitian_tiled(host, qubits);
    else bench_init_hermitian_packed(host, qubits);
    const int rc = orkan_state_upload(c->state, host);
    free(host);
    if (rc) { b200_cleanup(c); return NULL; }
    c->par = par;
    c->apply = b200_resolve(gate);
    return c;
}

static void *b200_tiled_init(qubit_t qubits, bench_gate_id_t gate, double par) {
    return b200_init(MIXED_TILED, qubits, gate, par);
}
static void *b200_packed_init(qubit_t qubits, bench_gate_id_t gate, double par) {
    return b200_init(MIXED_PACKED, qubits, gate, par);
}

static size_t b200_tiled_bytes(qubit_t qubits) {
    const idx_t dim = (idx_t)1 << qubits;
    if (qubits < LOG_TILE_DIM) return 2 * (size_t)dim * (size_t)dim * sizeof(cplx_t);
    const idx_t n_tiles = (dim + TILE_DIM - 1) / TILE_DIM;
    return 2 * (size_t)(n_tiles * (n_tiles + 1) / 2) * TILE_SIZE * sizeof(cplx_t);
}
static size_t b200_packed_bytes(qubit_t qubits) {
    const idx_t dim = (idx_t)1 << qubits;
    return 2 * (size_t)(dim * (dim + 1) / 2) * sizeof(cplx_t);
}

/* The storage (half of the touched bytes) must fit in free device memory. */
static int b200_fits(size_t touched) {
    size_t freeb = 0, totalb = 0;
    if (cudaMemGetInfo(&freeb, &totalb) != cudaSuccess) return 0;
    return touched / 2 < freeb;
}
static int b200_tiled_available(qubit_t qubits) { return b200_fits(b200_tiled_bytes(qubits)); }
static int b200_packed_available(qubit_t qubits) { return b200_fits(b200_packed_bytes(qubits)); }

const bench_backend_t orkan_b200_tiled_backend = {
    .name        = "orkan_b200_tiled",
    .init        = b200_tiled_init,
    .apply       = b200_apply,
    .cleanup     = b200_cleanup,
    .touch_bytes = b200_tiled_bytes,
    .available   = b200_tiled_available
};

const bench_backend_t orkan_b200_packed_backend = {
    .name        = "orkan_b200_packed",
    .init        = b200_packed_init,
    .apply       = b200_apply,
    .cleanup     = b200_cleanup,
    .touch_bytes = b200_packed_bytes,
    .available   = b200_packed_available
};

#ifdef BENCH_B200_AS_REFERENCE
extern const bench_backend_t orkan_tiled_backend __attribute__((alias("orkan_b200_tiled_backend")));
extern const bench_backend_t orkan_packed_backend __attribute__((alias("orkan_b200_packed_backend")));
#endif

#ifdef BENCH_B200_KRAUS
/* ---- Kraus benchmark ------------------------------------------------------------------ */
#include "channel.h"

typedef struct {
    state_t  *state;
    superop_t sop;
} b200_kraus_ctx_t;

static void b200_kraus_apply(void *ctx, const qubit_t *pos) {
    b200_kraus_ctx_t *c = (b200_kraus_ctx_t *)ctx;
    channel_1q(c->state, &c->sop, pos[0]);
    orkan_sync();
}

static void b200_kraus_cleanup(void *ctx) {
    b200_kraus_ctx_t *c = (b200_kraus_ctx_t *)ctx;
    state_free(c->state);
    free(c->state);
    free(c->sop.data);
    free(c);
}

static void *b200_kraus_init(state_type_t type, qubit_t qubits, int n_ops, int tgt_qubits, const cplx_t *ops) {
    if (tgt_qubits != 1) return NULL;                  /* channel_1q: 1-qubit channels, as the CPU version */
    b200_kraus_ctx_t *c = calloc(1, sizeof(b200_kraus_ctx_t));
    if (!c) return NULL;
    c->state = calloc(1, sizeof(state_t));
    if (!c->state) { free(c); return NULL; }
    c->state->type = type;
    state_init(c->state, qubits, NULL);
    if (!c->state->data) { free(c->state); free(c); return NULL; }
    const idx_t len = state_len(c->state);
    cplx_t *host = calloc(len, sizeof(cplx_t));
    if (!host) { state_free(c->state); free(c->state); free(c); return NULL; }
    if (type == MIXED_TILED) bench_init_hermitian_tiled(host, qubits);
    else bench_init_hermitian_packed(host, qubits);
    const int rc = orkan_state_upload(c->state, host);
    free(host);
    if (rc) { state_free(c->state); free(c->state); free(c); return NULL; }
    const kraus_t kraus = {(qubit_t)tgt_qubits, (uint64_t)n_ops, (cplx_t *)ops};
    c->sop = kraus_to_superop(&kraus);
    return c;
}

static void *b200_kraus_tiled_init(qubit_t q, int n_ops, int tgt, const cplx_t *ops) {
    return b200_kraus_init(MIXED_TILED, q, n_ops, tgt, ops);
}
static void *b200_kraus_packed_init(qubit_t q, int n_ops, int tgt, const cplx_t *ops) {
    return b200_kraus_init(MIXED_PACKED, q, n_ops, tgt, ops);
}

const bench_kraus_backend_t kraus_orkan_b200_tiled_backend = {
    .name        = "orkan_b200_tiled",
    .init        = b200_kraus_tiled_init,
    .apply       = b200_kraus_apply,
    .cleanup     = b200_kraus_cleanup,
    .touch_bytes = b200_tiled_bytes,
    .available   = b200_tiled_available
};

const bench_kraus_backend_t kraus_orkan_b200_packed_backend = {
    .name        = "orkan_b200_packed",
    .init        = b200_kraus_packed_init,
    .apply       = b200_kraus_apply,
    .cleanup     = b200_kraus_cleanup,
    .touch_bytes = b200_packed_bytes,
    .available   = b200_packed_available
};

#ifdef BENCH_B200_AS_REFERENCE
extern const bench_kraus_backend_t kraus_orkan_tiled_backend __attribute__((alias("kraus_orkan_b200_tiled_backend")));
extern const bench_kraus_backend_t kraus_orkan_packed_backend
    __attribute__((alias("kraus_orkan_b200_packed_backend")));
#endif
#endif /* BENCH_B200_KRAUS */
