/*
 * orkan_dev.h - extensions of the device build (no counterpart in the reference API,
 * which keeps state data in host memory and lets callers read state_t.data directly).
 */
#ifndef ORKAN_DEV_H
#define ORKAN_DEV_H

#include "state.h"
#include "channel.h"

#ifdef __cplusplus
extern "C" {
#endif

/* LOG_TILE_DIM this library was built with (the tiled layout's tile side is 2^value). */
int orkan_log_tile_dim(void);

/* Stream all calls are enqueued on (a cudaStream_t; NULL = the legacy default stream,
 * the initial setting).  Calls that return host values synchronise this stream. */
void orkan_set_stream(void *stream);
void *orkan_get_stream(void);

/* Wait until all work enqueued by the library on its stream has finished (queued
 * statevector gates are launched first). */
void orkan_sync(void);

/* Statevector gate fusion.  Gate calls on a PURE state join a queue, and consecutive gates
 * on the same statevector are applied in one pass over device memory.  Every other call
 * that touches device state launches the queue first, so results seen through the API are
 * those of the gates applied one by one (bit for bit).  Callers that read state_t.data with
 * their own kernels call orkan_flush (or orkan_sync) first, and callers that capture the
 * library stream into a CUDA graph call orkan_flush before they end the capture (queued
 * gates are launched at the flush).
 * orkan_set_gate_fusion(k) caps a fused run at k gates (at most 48); k <= 1 launches every
 * gate at once, as the reference applies it.  The initial cap is read from the environment
 * variable ORKAN_GATE_FUSION (default 48).  No counterpart in the reference. */
void orkan_flush(void);
void orkan_set_gate_fusion(unsigned max_gates);
unsigned orkan_get_gate_fusion(void);

/* Bulk copies of the whole storage (state_len(state) elements) between the device
 * state and a host buffer.  Return 0 on success, a cudaError_t value otherwise.
 * orkan_state_upload does not take ownership of host (compare state_init). */
int orkan_state_upload(state_t *state, const cplx_t *host);
int orkan_state_download(const state_t *state, cplx_t *host);

/* Asynchronous upload: enqueues the copy of host into the state's storage on stream (a
 * cudaStream_t; NULL: the library stream) and returns without waiting.  The copy starts after
 * all work enqueued so far on the library stream (queued gates are launched first), so work
 * that still reads or writes the state finishes before it is overwritten.  The caller keeps
 * host valid and unchanged until the copy has completed (pinned memory for a copy that
 * overlaps kernels), and orders later library work on the state after it, e.g. by making
 * the library stream wait for an event recorded on stream.  Returns 0 or a cudaError_t. */
int orkan_state_upload_async(state_t *state, const cplx_t *host, void *stream);

/* 2-qubit channel on a density matrix: sop from kraus_to_superop of 2-qubit Kraus operators
 * (16 x 16), local index 2 * bit(q0) + bit(q1).  The reference's channel_1q takes 1-local
 * superoperators only; this is its 2-local counterpart, with the same validation behaviour
 * ("orkan: channel: <msg>" and exit). */
void channel_2q(state_t *state, const superop_t *sop, qubit_t q0, qubit_t q1);

/* Cache of host observable / diagonal arrays (obs of mean and matel_diag, diag of
 * exp_diag).  Host arrays are copied to the device on every call by default.  With
 * orkan_set_host_array_cache(bytes), up to that many bytes of staged arrays stay on the
 * device, keyed by host pointer, length and a generation counter, so repeated calls with
 * the same array skip the copy.  A caller that changes a cached array in place must call
 * orkan_host_arrays_changed() before its next call (otherwise the stale device copy is
 * used).  orkan_set_host_array_cache(0) turns the cache off and frees it.  The statistics
 * count lookups that reused a copy (hits) and that staged one (misses). */
void orkan_set_host_array_cache(size_t max_bytes);
void orkan_host_arrays_changed(void);
void orkan_host_array_cache_stats(unsigned long long *hits, unsigned long long *misses);

/* Kernels launched by the library so far in this process. */
unsigned long long orkan_launch_count(void);

/* Test hook: make the next n device allocations of state storage fail, as an
 * out-of-memory device would (state_init / state_plus / state_cp then leave
 * data == NULL with a message on stderr, as the reference does on OOM). */
void orkan_debug_fail_allocs(int n);

#ifdef __cplusplus
}
#endif

#endif /* ORKAN_DEV_H */
