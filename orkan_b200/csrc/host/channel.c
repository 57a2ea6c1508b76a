/*
 * channel.c - superoperator construction (host) and 1-qubit channel application
 * (device).  Validation and messages follow reference src/channel/channel.c:8-85.
 */
#include "internal.h"

#include "channel.h"
#include "orkan_dev.h"

#define CHANNEL_VALIDATE(cond, msg) ORKAN_VALIDATE("channel", cond, msg)

/* S[(i,j),(k,l)] = sum_a K_a[i,k] conj(K_a[j,l]) with row index i*N + j and column
 * index k*N + l, K_a row-major (reference channel.c:21-50).  Returns calloc'd data
 * that the caller frees. */
superop_t kraus_to_superop(const kraus_t *kraus) {
    CHANNEL_VALIDATE(kraus && kraus->data, "kraus_to_superop: null kraus or data");
    const idx_t N = (idx_t)1 << kraus->n_qubits;
    const idx_t M = N * N;
    superop_t out = {0};
    out.n_qubits = kraus->n_qubits;
    out.data = calloc(M * M, sizeof(cplx_t));
    CHANNEL_VALIDATE(out.data, "kraus_to_superop: allocation failed");
    for (uint64_t a = 0; a < kraus->n_terms; ++a) {
        const cplx_t *K = kraus->data + a * M;
        for (idx_t i = 0; i < N; ++i)
            for (idx_t j = 0; j < N; ++j)
                for (idx_t k = 0; k < N; ++k)
                    for (idx_t l = 0; l < N; ++l)
                        out.data[(i * N + j) * M + (k * N + l)] += K[i * N + k] * conj(K[j * N + l]);
    }
    return out;
}

void channel_packed_1q(state_t *state, const cplx_t *sop, const qubit_t target) {
    orkan_check_cu("channel", "channel_1q",
                   orkan_cu_dm_superop1(MIXED_PACKED, LOG_TILE_DIM, state->data, state->qubits, target,
                                        (const double *)sop, orkan_stream()));
}

void channel_tiled_1q(state_t *state, const cplx_t *sop, const qubit_t target) {
    orkan_check_cu("channel", "channel_1q",
                   orkan_cu_dm_superop1(MIXED_TILED, LOG_TILE_DIM, state->data, state->qubits, target,
                                        (const double *)sop, orkan_stream()));
}

void channel_1q(state_t *state, const superop_t *sop, const qubit_t target) {
    CHANNEL_VALIDATE(state && state->data, "channel_1q: null state or data pointer");
    CHANNEL_VALIDATE(target < state->qubits, "channel_1q: target qubit out of range");
    CHANNEL_VALIDATE(sop && sop->data, "channel_1q: null superoperator or data pointer");
    CHANNEL_VALIDATE(sop->n_qubits == 1, "channel_1q: superoperator is not 1-local");
    switch (state->type) {
        case PURE:
            CHANNEL_VALIDATE(0, "channel_1q: not available for pure states");
            break;
        case MIXED_PACKED:
            channel_packed_1q(state, sop->data, target);
            break;
        case MIXED_TILED:
            channel_tiled_1q(state, sop->data, target);
            break;
        default:
            CHANNEL_VALIDATE(0, "channel_1q: unknown state type");
    }
}

/* 2-qubit channel (extension, include/orkan_dev.h): the reference's channel_1q accepts
 * 1-local superoperators only (channel.c:67-85), although kraus_to_superop builds them for
 * any qubit count.  Local index 2 * bit(q0) + bit(q1); vec index 4 * row + column. */
void channel_2q(state_t *state, const superop_t *sop, const qubit_t q0, const qubit_t q1) {
    CHANNEL_VALIDATE(state && state->data, "channel_2q: null state or data pointer");
    CHANNEL_VALIDATE(q0 < state->qubits && q1 < state->qubits, "channel_2q: qubit out of range");
    CHANNEL_VALIDATE(q0 != q1, "channel_2q: q0 and q1 must differ");
    CHANNEL_VALIDATE(sop && sop->data, "channel_2q: null superoperator or data pointer");
    CHANNEL_VALIDATE(sop->n_qubits == 2, "channel_2q: superoperator is not 2-local");
    CHANNEL_VALIDATE(state->type == MIXED_PACKED || state->type == MIXED_TILED,
                     "channel_2q: not available for pure states");
    orkan_check_cu("channel", "channel_2q",
                   orkan_cu_dm_superop2((int)state->type, LOG_TILE_DIM, state->data, state->qubits, q0, q1,
                                        (const double *)sop->data, orkan_stream()));
}
