/*
 * sample.c - sample_matrix (include/orkan_sample.h), the variational sample matrix that the
 * reference specifies in docs/SAMPLE_MATRIX.md and does not implement.
 *
 * The algorithm follows the specification's recommended form (section 6): the channels
 * below `at` are applied once, in place, to the input state (prefix sharing); the leaves
 * |psi_a> are built in column blocks of B vectors chosen from the workspace budget
 * (streaming); each diagonal block is reduced against itself and every later block against
 * it.  Channel sums sum_m w[m] M[m] x use two scratch vectors (copy, operate, accumulate).
 * All device memory is allocated on entry and freed on return.  The blocks of S come from
 * orkan_cu_sm_block, whose entries do not depend on the block shape, so the result is the
 * same for every budget.
 */
#include "internal.h"

#include <cuda_runtime.h>
#include <string.h>

#include "orkan_sample.h"

#define SM_VALIDATE(cond, msg) ORKAN_VALIDATE("sample_matrix", cond, msg)

enum { SM_TILE = 16 };

typedef struct {
    qubit_t n;
    size_t len;          /* amplitudes per vector */
    cplx_t *tmp, *acc;   /* channel-sum scratch */
    void *stream;
} sm_ctx_t;

static void sm_copy(const sm_ctx_t *c, cplx_t *dst, const cplx_t *src) {
    orkan_check_cu("sample_matrix", "copy",
                   (int)cudaMemcpyAsync(dst, src, c->len * sizeof(cplx_t), cudaMemcpyDeviceToDevice,
                                        (cudaStream_t)c->stream));
}

/* Run one operation on the vector x through a PURE state view of it. */
static void sm_run_op(const sm_ctx_t *c, qop_t op, cplx_t *x) {
    state_t view;
    view.type = PURE;
    view.data = x;
    view.qubits = c->n;
    op(&view);
    orkan_flush();                               /* the op's gates land before x is read */
    SM_VALIDATE(view.data == x && view.type == PURE && view.qubits == c->n,
                "an operation replaced, freed or resized the state's storage");
}

/* x <- sum_m w[m] ops[m] x, in place. */
static void sm_apply_channel(const sm_ctx_t *c, const sm_channel_t *ch, cplx_t *x) {
    for (unsigned m = 0; m < ch->n_ops; ++m) {
        sm_copy(c, c->tmp, x);
        sm_run_op(c, ch->ops[m], c->tmp);
        const double *w = (const double *)&ch->weights[m];
        orkan_check_cu("sample_matrix", "channel sum",
                       orkan_cu_lincomb(c->acc, c->tmp, w[0], w[1], c->len, m == 0, c->stream));
    }
    sm_copy(c, x, c->acc);
}

/* Leaves first .. first + count - 1 into dst (column k at dst + k len). */
static void sm_build_leaves(const sm_ctx_t *c, const cplx_t *prefix, const sm_channel_t *channels,
                            unsigned n_channels, unsigned at, unsigned first, unsigned count, cplx_t *dst) {
    for (unsigned k = 0; k < count; ++k) {
        cplx_t *x = dst + (size_t)k * c->len;
        sm_copy(c, x, prefix);
        sm_run_op(c, channels[at].ops[first + k], x);
        for (unsigned l = at + 1; l < n_channels; ++l) sm_apply_channel(c, &channels[l], x);
    }
}

/* Entries S[row, col] with row > col (and row == col: real part) of the block rows
 * r0 .. r0 + nr - 1 (vectors at pr) against columns c0 .. c0 + nc - 1 (vectors at pc). */
static void sm_reduce(const sm_ctx_t *c, const double *dobs, void *scratch, cplx_t *dout, cplx_t *hout,
                      const cplx_t *pr, unsigned r0, unsigned nr, const cplx_t *pc, unsigned c0, unsigned nc,
                      int diagonal_block, cplx_t *S, unsigned K) {
    for (unsigned tj = 0; tj < nc; tj += SM_TILE) {
        for (unsigned ti = diagonal_block ? tj : 0; ti < nr; ti += SM_TILE) {
            const unsigned bi = nr - ti < SM_TILE ? nr - ti : SM_TILE;
            const unsigned bj = nc - tj < SM_TILE ? nc - tj : SM_TILE;
            orkan_check_cu("sample_matrix", "block",
                           orkan_cu_sm_block(pr + (size_t)ti * c->len, bi, pc + (size_t)tj * c->len, bj, c->len,
                                             dobs, dout, scratch, c->stream));
            orkan_check_cu("sample_matrix", "block read-back",
                           (int)cudaMemcpyAsync(hout, dout, (size_t)bi * bj * sizeof(cplx_t),
                                                cudaMemcpyDeviceToHost, (cudaStream_t)c->stream));
            orkan_check_cu("sample_matrix", "synchronise", (int)cudaStreamSynchronize((cudaStream_t)c->stream));
            for (unsigned j = 0; j < bj; ++j) {
                for (unsigned i = 0; i < bi; ++i) {
                    const unsigned row = r0 + ti + i, col = c0 + tj + j;
                    const cplx_t v = hout[i + (size_t)j * bi];
                    if (row > col) S[row + (size_t)col * K] = v;
                    else if (row == col) S[row + (size_t)col * K] = creal(v);
                }
            }
        }
    }
}

void sample_matrix(state_t *iota, const double *obs, const sm_channel_t *channels, unsigned n_channels,
                   unsigned at, size_t workspace_bytes, cplx_t *S) {
    SM_VALIDATE(iota && iota->data, "null state or data pointer");
    SM_VALIDATE(iota->type == PURE, "the state must be PURE");
    SM_VALIDATE(obs, "null observable pointer");
    SM_VALIDATE(channels && n_channels > 0, "no channels");
    SM_VALIDATE(at < n_channels, "channel index out of range");
    SM_VALIDATE(S, "null output pointer");
    orkan_flush();
    for (unsigned l = 0; l < n_channels; ++l) {
        SM_VALIDATE(channels[l].n_ops > 0 && channels[l].ops, "a channel without operations");
        for (unsigned m = 0; m < channels[l].n_ops; ++m) SM_VALIDATE(channels[l].ops[m], "null operation");
        SM_VALIDATE(l == at || channels[l].weights, "null weights at a channel other than the chosen one");
    }
    sm_ctx_t c;
    c.n = iota->qubits;
    c.len = (size_t)1 << c.n;
    c.stream = orkan_stream();
    const size_t vec = c.len * sizeof(cplx_t);
    const unsigned K = channels[at].n_ops;
    /* budget: two channel-sum vectors + one block of K leaves, or two blocks of B */
    const size_t nvec = workspace_bytes / vec;
    unsigned B;
    int single;
    if (nvec >= 2 + (size_t)K) {
        B = K;
        single = 1;
    } else {
        SM_VALIDATE(nvec >= 4, "workspace too small: at least four state vectors of 2^n amplitudes are needed");
        const size_t b = (nvec - 2) / 2;
        B = (unsigned)(b < K ? b : K);
        single = 0;
    }
    const size_t scratch_cplx = (orkan_cu_sm_scratch_bytes() + sizeof(cplx_t) - 1) / sizeof(cplx_t);
    c.tmp = orkan_alloc_state(c.len);
    c.acc = orkan_alloc_state(c.len);
    cplx_t *phi_j = orkan_alloc_state((idx_t)c.len * B);
    cplx_t *phi_i = single ? NULL : orkan_alloc_state((idx_t)c.len * B);
    cplx_t *dobs_buf = orkan_alloc_state((c.len + 1) / 2);           /* 2^n doubles */
    cplx_t *scratch = orkan_alloc_state(scratch_cplx);
    cplx_t *dout = orkan_alloc_state(SM_TILE * SM_TILE);
    cplx_t *hout = (cplx_t *)malloc(SM_TILE * SM_TILE * sizeof(cplx_t));
    if (!c.tmp || !c.acc || !phi_j || (!single && !phi_i) || !dobs_buf || !scratch || !dout || !hout) {
        orkan_free_device(c.tmp);
        orkan_free_device(c.acc);
        orkan_free_device(phi_j);
        orkan_free_device(phi_i);
        orkan_free_device(dobs_buf);
        orkan_free_device(scratch);
        orkan_free_device(dout);
        free(hout);
        SM_VALIDATE(0, "device allocation failed");
    }
    double *dobs = (double *)dobs_buf;
    orkan_check_cu("sample_matrix", "observable upload",
                   (int)cudaMemcpyAsync(dobs, obs, c.len * sizeof(double), cudaMemcpyDefault, (cudaStream_t)c.stream));
    /* prefix: K_{at-1} ... K_0 |iota>, once, in the caller's buffer */
    for (unsigned l = 0; l < at; ++l) sm_apply_channel(&c, &channels[l], iota->data);
    for (unsigned jb = 0; jb < K; jb += B) {
        const unsigned bj = K - jb < B ? K - jb : B;
        sm_build_leaves(&c, iota->data, channels, n_channels, at, jb, bj, phi_j);
        sm_reduce(&c, dobs, scratch, dout, hout, phi_j, jb, bj, phi_j, jb, bj, 1, S, K);
        for (unsigned ib = jb + bj; ib < K; ib += B) {
            const unsigned bi = K - ib < B ? K - ib : B;
            sm_build_leaves(&c, iota->data, channels, n_channels, at, ib, bi, phi_i);
            sm_reduce(&c, dobs, scratch, dout, hout, phi_i, ib, bi, phi_j, jb, bj, 0, S, K);
        }
    }
    for (unsigned j = 0; j < K; ++j)
        for (unsigned i = j + 1; i < K; ++i) S[j + (size_t)i * K] = conj(S[i + (size_t)j * K]);
    orkan_check_cu("sample_matrix", "synchronise", (int)cudaStreamSynchronize((cudaStream_t)c.stream));
    orkan_free_device(c.tmp);
    orkan_free_device(c.acc);
    orkan_free_device(phi_j);
    orkan_free_device(phi_i);
    orkan_free_device(dobs_buf);
    orkan_free_device(scratch);
    orkan_free_device(dout);
    free(hout);
}
