/* orkan_sample.h - the variational sample matrix on device-resident statevectors.
 *
 * The reference specifies this operation but does not implement it
 * (docs/SAMPLE_MATRIX.md: definition section 1, inputs 2, output 3, memory requirements 4,
 * recommended algorithm 6); this library provides it.  For an ansatz of channels
 * K_l = sum_m w_l[m] M_l[m] applied to |iota>, and a channel index l*, it returns the
 * K x K Hermitian matrix
 *     S[a, b] = <psi_a| diag(obs) |psi_b>,
 *     |psi_a> = K_{L-1} ... K_{l*+1} M_{l*}[a] K_{l*-1} ... K_0 |iota>.
 */
#ifndef ORKAN_SAMPLE_H
#define ORKAN_SAMPLE_H

#include <stddef.h>

#include "q_types.h"
#include "state.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One channel of the ansatz: sum_m weights[m] * ops[m].  An operation is a qop_t that
 * applies gates of this library to the PURE state it is given, in place; it must not
 * free, replace or resize the state's storage.  weights may be NULL for the channel at
 * which the sample matrix is taken (it is not used there). */
typedef struct {
    unsigned n_ops;
    const qop_t *ops;
    const cplx_t *weights;
} sm_channel_t;

/* S^(at) of the ansatz channels[0 .. n_channels) applied to iota (0-based channel index
 * `at`), written column-major into the caller's host buffer S (K x K, K = channels[at].n_ops,
 * S[i + j K] = S_ij): both triangles filled, S_ji = conj(S_ij) exactly, diagonal imaginary
 * parts exactly zero.  obs: 2^n doubles (host or device pointer).
 *
 * iota must be PURE; it is consumed: on return it holds K_{at-1} ... K_0 |iota>, computed
 * once for all columns.  workspace_bytes caps the device scratch held at once: two state
 * vectors for the channel sums plus two blocks of B leaf vectors (one block of K when it
 * fits), B chosen from the budget; at least four state vectors of 2^n amplitudes are
 * needed.  All scratch is allocated on entry and freed on return.  The result does not
 * depend on the budget (bit for bit): every entry is the same fixed-order reduction.
 * Invalid arguments, a budget below four vectors, an operation that changes the state's
 * storage and allocation failures print "orkan: sample_matrix: <msg>" and exit, as the
 * reference's validation does. */
void sample_matrix(state_t *iota, const double *obs, const sm_channel_t *channels, unsigned n_channels,
                   unsigned at, size_t workspace_bytes, cplx_t *S);

#ifdef __cplusplus
}
#endif

#endif /* ORKAN_SAMPLE_H */
