/*
 * fuse.c - the statevector gate queue.
 *
 * The reference applies every gate call as its own pass over the state
 * (src/gate/gate_pure.c:33-48).  Here the 18 gate calls on a PURE state do not launch at
 * once: they join a queue, and consecutive gates on the same statevector are applied
 * together by orkan_cu_pure_fused, one pass over HBM for the whole run.  A gate can join
 * while the qubits the run mixes (targets of X/Y/H/Hy/Rx/Ry/CX/CY/CCX, both qubits of
 * SWAP), together with qubits 0-2, fit the chunk of 2^C amplitudes (C = n up to 12 qubits,
 * else 11); controls and diagonal gates can always join.
 *
 * The queue is flushed (its gates launched, in order, on the library stream) before any
 * other call that touches device state: state_* functions, mean, matel_diag, exp_diag,
 * channels, density-matrix gates, sample_matrix, the bulk copies, orkan_sync and a change
 * of stream.  So every result a caller can observe through the API is the one of the gates
 * applied one by one (bit for bit: the fused kernel uses the per-gate arithmetic).  A
 * caller that reads state_t.data with its own kernels calls orkan_flush (or orkan_sync)
 * first.  state_free drops the queue of the state it frees.
 *
 * orkan_set_gate_fusion(k) caps a run at k gates (k <= 1: every gate launches at once, the
 * reference's behaviour); the initial cap comes from the environment variable
 * ORKAN_GATE_FUSION (default 48).  A mutex serialises the queue between host threads.
 */
#include "internal.h"

#include <pthread.h>

#define FUSE_MAX 48u

static pthread_mutex_t g_fuse_mu = PTHREAD_MUTEX_INITIALIZER;
static int g_fuse_cap = -1;          /* -1: not yet read from the environment */
static int g_fuse_log_chunk = -1;

static struct {
    cplx_t *data;
    unsigned n, log_chunk, count;
    unsigned long long need;         /* qubits the run holds local */
    orkan_fgate_t g[FUSE_MAX];
} Q;

static unsigned fuse_cap(void) {
    if (g_fuse_cap < 0) {
        const char *e = getenv("ORKAN_GATE_FUSION");
        int v = e ? atoi(e) : (int)FUSE_MAX;
        g_fuse_cap = v < 0 ? 0 : (v > (int)FUSE_MAX ? (int)FUSE_MAX : v);
    }
    return (unsigned)g_fuse_cap;
}

/* Chunk size of a run on n qubits: the whole state up to 12 qubits (one block holds it),
 * 2^11 amplitudes above (environment variable ORKAN_FUSE_LOG_CHUNK, 5..12, overrides). */
static unsigned fuse_log_chunk(unsigned n) {
    if (g_fuse_log_chunk < 0) {
        const char *e = getenv("ORKAN_FUSE_LOG_CHUNK");
        int v = e ? atoi(e) : 0;
        g_fuse_log_chunk = (v >= 5 && v <= 12) ? v : 0;
    }
    if (g_fuse_log_chunk > 0) return n < (unsigned)g_fuse_log_chunk ? n : (unsigned)g_fuse_log_chunk;
    return n <= 12 ? n : 11u;
}

static int popcount64(unsigned long long x) { return __builtin_popcountll(x); }

/* One gate through its own kernel. */
static int launch_one(cplx_t *data, unsigned n, const orkan_fgate_t *g) {
    void *st = orkan_stream();
    switch (g->op) {
        case ORKAN_FOP_CX: return orkan_cu_pure_gate2(data, n, g->q[0], g->q[1], ORKAN_OP_CX, st);
        case ORKAN_FOP_CY: return orkan_cu_pure_gate2(data, n, g->q[0], g->q[1], ORKAN_OP_CY, st);
        case ORKAN_FOP_CZ: return orkan_cu_pure_gate2(data, n, g->q[0], g->q[1], ORKAN_OP_CZ, st);
        case ORKAN_FOP_SWAP: return orkan_cu_pure_gate2(data, n, g->q[0], g->q[1], ORKAN_OP_SWAP, st);
        case ORKAN_FOP_CCX: return orkan_cu_pure_ccx(data, n, g->q[0], g->q[1], g->q[2], st);
        default: return orkan_cu_pure_gate1(data, n, g->q[0], g->op, g->c, g->s, st);
    }
}

static void flush_locked(void) {
    if (!Q.count) return;
    const int rc = Q.count == 1 ? launch_one(Q.data, Q.n, &Q.g[0])
                                : orkan_cu_pure_fused(Q.data, Q.n, Q.log_chunk, Q.count, Q.g, orkan_stream());
    Q.count = 0;
    Q.data = NULL;
    Q.need = 0;
    orkan_check_cu("gate", "queued gates", rc);
}

void orkan_flush(void) {
    pthread_mutex_lock(&g_fuse_mu);
    flush_locked();
    pthread_mutex_unlock(&g_fuse_mu);
}

void orkan_fuse_drop(const void *data) {
    pthread_mutex_lock(&g_fuse_mu);
    if (Q.count && Q.data == data) {
        Q.count = 0;
        Q.data = NULL;
        Q.need = 0;
    }
    pthread_mutex_unlock(&g_fuse_mu);
}

void orkan_set_gate_fusion(unsigned max_gates) {
    pthread_mutex_lock(&g_fuse_mu);
    flush_locked();
    g_fuse_cap = (int)(max_gates > FUSE_MAX ? FUSE_MAX : max_gates);
    pthread_mutex_unlock(&g_fuse_mu);
}

unsigned orkan_get_gate_fusion(void) {
    pthread_mutex_lock(&g_fuse_mu);
    const unsigned v = fuse_cap();
    pthread_mutex_unlock(&g_fuse_mu);
    return v;
}

void orkan_pure_gate(state_t *state, const orkan_fgate_t *g, const char *name) {
    const unsigned n = state->qubits;
    pthread_mutex_lock(&g_fuse_mu);
    const unsigned cap = fuse_cap();
    if (cap <= 1) {
        flush_locked();
        pthread_mutex_unlock(&g_fuse_mu);
        orkan_check_cu("gate", name, launch_one(state->data, n, g));
        return;
    }
    if (Q.count && (Q.data != state->data || Q.n != n)) flush_locked();
    const unsigned lc = fuse_log_chunk(n);
    const unsigned long long low = n >= 3 ? 7ull : ((1ull << n) - 1ull);
    const unsigned long long need = orkan_cu_fused_need(g) | low;
    if (Q.count && (popcount64(Q.need | need) > (int)lc || Q.count >= cap)) flush_locked();
    if (popcount64(need) > (int)lc) {            /* cannot be fused at all: launch now */
        pthread_mutex_unlock(&g_fuse_mu);
        orkan_check_cu("gate", name, launch_one(state->data, n, g));
        return;
    }
    if (!Q.count) {
        Q.data = state->data;
        Q.n = n;
        Q.log_chunk = lc;
        Q.need = 0;
    }
    Q.need |= need;
    Q.g[Q.count++] = *g;
    pthread_mutex_unlock(&g_fuse_mu);
}
