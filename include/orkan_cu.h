/*
 * orkan_cu.h - C-ABI of the sm_100a kernel layer.
 *
 * Plain C types only (no CUDA, torch or C99-complex types in the signatures): device
 * buffers are void*, complex coefficient arrays are interleaved (re, im) doubles,
 * streams are cudaStream_t passed as void* (NULL = the legacy default stream).
 * Every function enqueues its kernel(s) on the stream and returns 0, or a nonzero
 * cudaError_t value (launch failure, invalid argument).  Functions that return a
 * value to the host (orkan_cu_mean, orkan_cu_matel_diag) return once the value is
 * available: all work enqueued on the stream before them has then completed (the
 * reduction's own launch may still be retiring).
 *
 * Layout codes follow state_type_t: 0 = PURE, 1 = MIXED_PACKED, 2 = MIXED_TILED;
 * log_tile is the LOG_TILE_DIM of the tiled layout (ignored otherwise).
 * Local-index convention for k-qubit operators: qubits[0] is the most significant
 * bit of the 2^k-dimensional local index (the reference test convention,
 * test/utility/gatemat.c:178-181).
 *
 * The public Orkan API (state.h, gate.h, channel.h, meas.h, circ.h) is implemented on
 * top of these calls; each entry below names the reference backends it replaces.
 */
#ifndef ORKAN_CU_H
#define ORKAN_CU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* PURE 1-qubit op codes (order of reference include/gate.h:28-49). */
enum orkan_op1 {
    ORKAN_OP_X = 0, ORKAN_OP_Y, ORKAN_OP_Z, ORKAN_OP_H, ORKAN_OP_S, ORKAN_OP_SDG,
    ORKAN_OP_T, ORKAN_OP_TDG, ORKAN_OP_HY, ORKAN_OP_RX, ORKAN_OP_RY, ORKAN_OP_RZ, ORKAN_OP_P
};
/* PURE 2-qubit op codes. */
enum orkan_op2 { ORKAN_OP_CX = 0, ORKAN_OP_CY, ORKAN_OP_CZ, ORKAN_OP_SWAP };

/* Fill every live stored element with (re, im); the tiled padding of 2^n < TILE_DIM
 * stays untouched.  Replaces the fill loops of state_pure_plus / state_packed_plus /
 * state_tiled_plus (reference src/state/state_pure.c:30-43, state_packed.c:57-76,
 * state_tiled.c:84-114). */
int orkan_cu_fill(int layout, unsigned log_tile, void *data, unsigned n, double re, double im, void *stream);

/* 1-qubit gate on a statevector: op in orkan_op1; c, s as the reference host code
 * computes them (cos/sin of theta/2 for RX/RY/RZ, of theta for P; ignored otherwise).
 * Replaces x_pure ... p_pure (reference src/gate/gate_pure.c:125-268). */
int orkan_cu_pure_gate1(void *psi, unsigned n, unsigned target, int op, double c, double s, void *stream);

/* CX / CY / CZ (qa = control, qb = target) or SWAP (qa, qb) on a statevector.
 * Replaces cx_pure / cy_pure / cz_pure / swap_pure (reference gate_pure.c:282-396). */
int orkan_cu_pure_gate2(void *psi, unsigned n, unsigned qa, unsigned qb, int op, void *stream);

/* Toffoli on a statevector.  Replaces ccx_pure (reference gate_pure.c:405-434). */
int orkan_cu_pure_ccx(void *psi, unsigned n, unsigned c1, unsigned c2, unsigned t, void *stream);

/* A run of statevector gates applied in one pass over the amplitudes.  Gate codes: the
 * orkan_op1 codes (q[0] = target; c, s as for orkan_cu_pure_gate1) and the orkan_fop codes
 * (CX/CY: q[0] control, q[1] target; CZ and SWAP: q[0], q[1]; CCX: q[0], q[1] controls,
 * q[2] target).  The state is cut into chunks of 2^log_chunk amplitudes that differ in
 * log_chunk "local" qubits: qubits 0-2 and every qubit a gate of the run mixes (the target
 * of X/Y/H/Hy/Rx/Ry/CX/CY/CCX, both qubits of SWAP), filled up with the lowest free qubits.
 * Each chunk is loaded once, every gate is applied to it in shared memory with the
 * arithmetic of the one-gate kernels (bit-identical results), and it is stored once.
 * No counterpart in the reference, which makes one pass per gate
 * (src/gate/gate_pure.c:33-48 and :282-434).  1 <= ngates <= 48, log_chunk <= min(n, 12). */
enum orkan_fop { ORKAN_FOP_CX = 16, ORKAN_FOP_CY, ORKAN_FOP_CZ, ORKAN_FOP_SWAP, ORKAN_FOP_CCX };
typedef struct {
    int op;
    unsigned q[3];
    double c, s;
} orkan_fgate_t;

int orkan_cu_pure_fused(void *psi, unsigned n, unsigned log_chunk, unsigned ngates, const orkan_fgate_t *gates,
                        void *stream);

/* The qubits gate g mixes (which a fused run must hold local), as a bit mask; all bits set
 * for an invalid op code. */
unsigned long long orkan_cu_fused_need(const orkan_fgate_t *g);

/* rho -> U rho U^dagger for a dense k-qubit U (k = 1 or 2), u = 2^k x 2^k row-major
 * interleaved complex.  Replaces h/hy/rx/ry_{packed,tiled} and the generic
 * single_from_mat / two_from_mat (reference gate_packed_1q.c:126-677,
 * gate_tiled_{h,hy,rx,ry}.c, gate_tiled_1q.c:3-184, gate_tiled_2q.c:3). */
int orkan_cu_dm_unitary(int layout, unsigned log_tile, void *rho, unsigned n, unsigned k,
                        const unsigned *qubits, const double *u, void *stream);

/* rho -> U rho U^dagger for a monomial U with involutive permutation:
 * (U psi)[y] = phase[y] psi[src[y]] on the k-qubit local index (k = 1..3), src[src[y]] == y.
 * Replaces x/y_{packed,tiled}, cx/cy/swap/ccx_{packed,tiled} (reference
 * gate_packed_{cx,cy,swap,ccx}.c, gate_tiled_{x,y,cx,cy,swap,ccx}.c). */
int orkan_cu_dm_monomial(int layout, unsigned log_tile, void *rho, unsigned n, unsigned k,
                         const unsigned *qubits, const unsigned *src, const double *phase, void *stream);

/* rho_rc *= phi(r) conj(phi(c)) for a diagonal k-qubit gate phi(x) = phase[local(x)]
 * (k = 1..3).  Replaces z/s/sdg/t/tdg/p/rz_{packed,tiled} and cz_{packed,tiled}
 * (reference gate_packed_1q.c:481-523, gate_packed_cz.c:23-80, gate_tiled_{z,s,t,p,rz,cz}.c). */
int orkan_cu_dm_phase(int layout, unsigned log_tile, void *rho, unsigned n, unsigned k,
                      const unsigned *qubits, const double *phase, void *stream);

/* 1-qubit channel: vec(rho_2x2)' = sop vec(rho_2x2), sop 4x4 row-major interleaved
 * complex, vec order (00, 01, 10, 11).  Replaces channel_packed_1q / channel_tiled_1q
 * (reference src/channel/channel_packed.c:48-120, channel_tiled.c:52-185). */
int orkan_cu_dm_superop1(int layout, unsigned log_tile, void *rho, unsigned n, unsigned target,
                         const double *sop, void *stream);

/* 2-qubit superoperator on (q0, q1): sop = 16 x 16 row-major complex over vec(rho_4x4) with
 * vec index 4 * row + column and local index 2 * bit(q0) + bit(q1).  No counterpart in the
 * reference, whose channel_1q takes 1-local superoperators only (src/channel/channel.c:67-85)
 * although kraus_to_superop builds them for any qubit count (channel.c:21-50). */
int orkan_cu_dm_superop2(int layout, unsigned log_tile, void *rho, unsigned n, unsigned q0, unsigned q1,
                         const double *sop, void *stream);

/* exp_diag with a DEVICE diag array of 2^n doubles.  Replaces exp_diag_pure /
 * exp_diag_packed / exp_diag_tiled (reference src/circ/circ_pure.c:21-33,
 * circ_packed.c:28-71, circ_tiled.c:25-105).  t == 0 is a no-op. */
int orkan_cu_exp_diag(int layout, unsigned log_tile, void *data, unsigned n, const double *diag,
                      double t, void *stream);

/* mean with a DEVICE obs array; *result receives the value (host pointer).  Replaces
 * mean_pure / mean_packed / mean_tiled (reference src/meas/meas_pure.c:20-30,
 * meas_packed.c:23-51, meas_tiled.c:29-69). */
int orkan_cu_mean(int layout, unsigned log_tile, const void *data, unsigned n, const double *obs,
                  double *result, void *stream);

/* matel_diag on statevectors with a DEVICE obs array; result[0..1] = (re, im).
 * Replaces matel_diag_pure (reference src/meas/meas_pure.c:32-46). */
int orkan_cu_matel_diag(const void *bra, const void *ket, unsigned n, const double *obs,
                        double *result, void *stream);

/* exp_diag on a MIXED_PACKED (layout 1) or MIXED_TILED (layout 2) density matrix that
 * allocates nothing.  No counterpart in the reference: it exists for callers that cannot
 * let the library call cudaMalloc/cudaFree -- programs whose own pool allocator holds
 * nearly all device memory, and latency-sensitive callers that cannot absorb the
 * device-wide wait of cudaFree when orkan_cu_exp_diag grows its scratch buffer.
 * The per-index phase table lives in a fixed device array of 65536 entries (1 MiB per
 * device, kept until the library is unloaded): n > 16 is rejected with a message on
 * stderr and cudaErrorInvalidValue.  data and diag are caller-owned device buffers.  The
 * first call on a device resolves the array's device address (cudaGetSymbolAddress);
 * make that first call before any stream capture.  All calls on a device share the array
 * and it keeps the last call's contents; calls whose kernels overlap on the GPU race.
 * Same results as orkan_cu_exp_diag; t == 0 is a no-op. */
int orkan_cu_exp_diag_noalloc(int layout, unsigned log_tile, void *data, unsigned n, const double *diag,
                              double t, void *stream);

/* Error word of the density-matrix engine on the current device: 0, or bit 0 set when a
 * kernel's bounded wait for staged data ran out (the kernel then stopped early instead of
 * waiting forever).  Reads device memory, so it synchronises with the device. */
unsigned orkan_cu_engine_status(void);

/* Reset the engine's error word to 0 on the current device (synchronises). */
int orkan_cu_engine_status_clear(void);

/* Test hook of the failure path: polls > 0 limits each of the engine's waits for staged
 * data to that many polls (0 restores the default of 2^24); drop_loads != 0 (with polls > 0)
 * arms each item's completion barrier but issues none of its copies, so the wait runs out
 * with nothing in flight and the kernel returns early with bit 0 of the error word set.
 * The state's contents are unspecified after such a launch.  Not for production use. */
void orkan_cu_engine_test_wait(unsigned long long polls, int drop_loads);

/* Number of kernels this library has launched in this process (all devices). */
unsigned long long orkan_cu_launch_count(void);

/* ---- sample-matrix building blocks (sample_matrix, include/orkan_sample.h; the reference
 * specifies the operation in docs/SAMPLE_MATRIX.md and has no implementation) ---------- */

/* acc = w x (first != 0) or acc += w x over len amplitudes (w = w_re + i w_im). */
int orkan_cu_lincomb(void *acc, const void *x, double w_re, double w_im, unsigned long long len, int first,
                     void *stream);

/* Bytes of device scratch orkan_cu_sm_block needs (fixed; about 2 MiB). */
size_t orkan_cu_sm_scratch_bytes(void);

/* out[i + j bi] = sum_x conj(phi_i[i len + x]) obs[x] phi_j[j len + x] for i < bi, j < bj
 * (1 <= bi, bj <= 16; columns of len amplitudes, consecutive).  The sum over x runs in a
 * fixed partition and order that depend only on len, so an entry is the same bit for bit
 * whatever block it is computed in. */
int orkan_cu_sm_block(const void *phi_i, unsigned bi, const void *phi_j, unsigned bj, unsigned long long len,
                      const double *obs, void *out, void *scratch, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* ORKAN_CU_H */
