/*
 * orkan_batch.h - batched QAOA-style diagonal-cost circuits (no counterpart in the
 * reference's API; each instance is the composition of reference calls):
 *
 *     state_plus(&s, n)                                  (reference src/state/state_pure.c:30-43)
 *     for k < p:  exp_diag(&s, cost, gamma[k])           (src/circ/circ_pure.c:21-33)
 *                 rx(&s, q, 2 * beta[k]) for q < n       (src/gate/gate_pure.c:230-234)
 *     result = mean(&s, cost)                            (src/meas/meas_pure.c:20-30)
 *
 * The cost of instance i is the weighted cut of its graph:
 *     cost(x) = sum over edges e = (u, v), in the given order, of w_e * [bit u of x != bit v of x]
 * (MaxCut; integer-valued and exact in FP64 for integer weights).  All instances of a batch
 * share p; their qubit counts may differ (1 <= n <= 26).  The batch is evaluated by one set of
 * fused passes per wave (p + 1 passes over every amplitude instead of (n + 1) p + 2), launched
 * from a CUDA graph captured at creation and replayed by every orkan_qaoa_run call.
 * Functions return 0 or a cudaError_t value.
 */
#ifndef ORKAN_BATCH_H
#define ORKAN_BATCH_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orkan_qaoa orkan_qaoa_t;

/* Creation flags. */
#define ORKAN_QAOA_F64_COSTS 1u   /* keep every cost vector in FP64 (default: integer costs
                                     below 256 are stored as bytes, which is exact) */

/* Create a batch of `count` instances on the current device.
 *   n_qubits[i]        qubits of instance i
 *   edge_offsets       count + 1 offsets into edges / weights (instance i: [off[i], off[i+1]))
 *   edges              2 * total vertex indices (u, v) of every edge, u, v < n_qubits[i], u != v
 *   weights            total weights, or NULL for unit weights
 *   p                  layers
 *   mem_budget         device bytes the batch may use for state vectors (0: 60 % of the free
 *                      memory after the cost vectors); instances are evaluated in waves that fit
 *   flags              ORKAN_QAOA_* flags
 * Instances with the same qubit count, edge list and weights share one resident cost vector
 * (2^n bytes for byte costs, plus a transposed copy of the same size that the high passes
 * read; 2^n doubles for FP64 costs).  All arrays are host arrays, copied. */
int orkan_qaoa_create(orkan_qaoa_t **out, unsigned count, const unsigned *n_qubits, const unsigned *edge_offsets,
                      const unsigned *edges, const double *weights, unsigned p, unsigned long long mem_budget,
                      unsigned flags);

/* Evaluate every instance: gammas and betas are host arrays [count][p] in instance order;
 * means[i] receives the expectation value of the cost.  Synchronises the stream. */
int orkan_qaoa_run(orkan_qaoa_t *b, const double *gammas, const double *betas, double *means, void *stream);

/* Autotune chunk size, block size and buffer depth per qubit count on this batch (timing
 * candidate launch plans on the device with the given angles), keep the fastest and rebuild
 * the graph.  When
 * cache_path is not NULL the choice is read from / stored in that JSON file, keyed by the
 * device name and the batch's qubit counts. */
int orkan_qaoa_tune(orkan_qaoa_t *b, const double *gammas, const double *betas, const char *cache_path);

/* Current launch configuration of instances of n qubits: log2 of the chunk (amplitudes per
 * work item), threads per block, and the number of shared buffers per block (2: the next
 * item is copied in while the current one computes). */
int orkan_qaoa_config(const orkan_qaoa_t *b, unsigned n, unsigned *log_chunk, unsigned *threads, unsigned *ring);

/* Copy the device cost vector of instance i (2^n doubles) to host memory (for checks). */
int orkan_qaoa_cost_vector(orkan_qaoa_t *b, unsigned i, double *host_out);

/* Waves, passes and kernel launches per orkan_qaoa_run. */
int orkan_qaoa_stats(const orkan_qaoa_t *b, unsigned *waves, unsigned *launches);

void orkan_qaoa_destroy(orkan_qaoa_t *b);

#ifdef __cplusplus
}
#endif

#endif /* ORKAN_BATCH_H */
