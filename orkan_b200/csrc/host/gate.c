/*
 * gate.c - the 18 gate calls: validation and layout dispatch in C (same checks and
 * messages as reference src/gate/gate.c:19-219), then one kernel launch through the
 * C-ABI of include/orkan_cu.h.
 *
 * Per-layout backends keep the reference's exported names (x_pure, x_packed, x_tiled,
 * ..., single_from_mat, two_from_mat) so harnesses that call them directly still link.
 *
 * Density-matrix gates are grouped by their structure:
 *   mixing    H, Hy, Rx, Ry, single_from_mat, two_from_mat -> orkan_cu_dm_unitary
 *   monomial  X, Y, CX, CY, SWAP, CCX                       -> orkan_cu_dm_monomial
 *   diagonal  Z, S, Sdg, T, Tdg, P, Rz, CZ                  -> orkan_cu_dm_phase
 * P and Rz act identically on a density matrix (phase e^{i theta} on rho_10 with
 * c = cos(theta), s = sin(theta)), as the reference notes at gate_tiled_p.c:1-22.
 */
#include "internal.h"

#include <math.h>

#define GATE_VALIDATE(cond, msg) ORKAN_VALIDATE("gate", cond, msg)

static const double R2 = 0.70710678118654752440;   /* M_SQRT1_2 */

/* ---- PURE backends: gates join the statevector gate queue (fuse.c) --------------- */
static void pure1(state_t *s, qubit_t q, int op, double c, double sn, const char *name) {
    const orkan_fgate_t g = {op, {q, 0, 0}, c, sn};
    orkan_pure_gate(s, &g, name);
}
static void pure2(state_t *s, qubit_t a, qubit_t b, int op, const char *name) {
    const orkan_fgate_t g = {op, {a, b, 0}, 0.0, 0.0};
    orkan_pure_gate(s, &g, name);
}

void x_pure(state_t *state, qubit_t target)   { pure1(state, target, ORKAN_OP_X, 0, 0, "x"); }
void y_pure(state_t *state, qubit_t target)   { pure1(state, target, ORKAN_OP_Y, 0, 0, "y"); }
void z_pure(state_t *state, qubit_t target)   { pure1(state, target, ORKAN_OP_Z, 0, 0, "z"); }
void h_pure(state_t *state, qubit_t target)   { pure1(state, target, ORKAN_OP_H, 0, 0, "h"); }
void s_pure(state_t *state, qubit_t target)   { pure1(state, target, ORKAN_OP_S, 0, 0, "s"); }
void sdg_pure(state_t *state, qubit_t target) { pure1(state, target, ORKAN_OP_SDG, 0, 0, "sdg"); }
void t_pure(state_t *state, qubit_t target)   { pure1(state, target, ORKAN_OP_T, 0, 0, "t"); }
void tdg_pure(state_t *state, qubit_t target) { pure1(state, target, ORKAN_OP_TDG, 0, 0, "tdg"); }
void hy_pure(state_t *state, qubit_t target)  { pure1(state, target, ORKAN_OP_HY, 0, 0, "hy"); }

/* host-side coefficients exactly as the reference computes them (gate_pure.c:190-268) */
void rx_pure(state_t *state, qubit_t target, double theta) {
    pure1(state, target, ORKAN_OP_RX, cos(theta / 2.0), sin(theta / 2.0), "rx");
}
void ry_pure(state_t *state, qubit_t target, double theta) {
    pure1(state, target, ORKAN_OP_RY, cos(theta / 2.0), sin(theta / 2.0), "ry");
}
void rz_pure(state_t *state, qubit_t target, double theta) {
    pure1(state, target, ORKAN_OP_RZ, cos(theta / 2.0), sin(theta / 2.0), "rz");
}
void p_pure(state_t *state, qubit_t target, double theta) {
    pure1(state, target, ORKAN_OP_P, cos(theta), sin(theta), "p");
}

void cx_pure(state_t *state, qubit_t control, qubit_t target) { pure2(state, control, target, ORKAN_FOP_CX, "cx"); }
void cy_pure(state_t *state, qubit_t control, qubit_t target) { pure2(state, control, target, ORKAN_FOP_CY, "cy"); }
void cz_pure(state_t *state, qubit_t control, qubit_t target) { pure2(state, control, target, ORKAN_FOP_CZ, "cz"); }
void swap_pure(state_t *state, qubit_t q1, qubit_t q2) { pure2(state, q1, q2, ORKAN_FOP_SWAP, "swap"); }
void ccx_pure(state_t *state, qubit_t ctrl1, qubit_t ctrl2, qubit_t target) {
    const orkan_fgate_t g = {ORKAN_FOP_CCX, {ctrl1, ctrl2, target}, 0.0, 0.0};
    orkan_pure_gate(state, &g, "ccx");
}

/* ---- density-matrix backends (packed and tiled share the kernels) ---------------- */
static void dm_mix1(state_t *s, qubit_t q, const double u[8], const char *name) {
    const unsigned qs[1] = {q};
    orkan_check_cu("gate", name,
                   orkan_cu_dm_unitary((int)s->type, LOG_TILE_DIM, s->data, s->qubits, 1, qs, u, orkan_stream()));
}

static void dm_mono(state_t *s, unsigned k, const unsigned *qs, const unsigned *src, const double *ph,
                    const char *name) {
    orkan_check_cu("gate", name,
                   orkan_cu_dm_monomial((int)s->type, LOG_TILE_DIM, s->data, s->qubits, k, qs, src, ph, orkan_stream()));
}

static void dm_phase1(state_t *s, qubit_t q, double re1, double im1, const char *name) {
    const unsigned qs[1] = {q};
    const double ph[4] = {1.0, 0.0, re1, im1};
    orkan_check_cu("gate", name,
                   orkan_cu_dm_phase((int)s->type, LOG_TILE_DIM, s->data, s->qubits, 1, qs, ph, orkan_stream()));
}

static void dm_x(state_t *s, qubit_t q) {
    const unsigned qs[1] = {q}, src[2] = {1, 0};
    const double ph[4] = {1, 0, 1, 0};
    dm_mono(s, 1, qs, src, ph, "x");
}
static void dm_y(state_t *s, qubit_t q) {
    /* Y|0> = i|1>, Y|1> = -i|0>:  (Y psi)[0] = -i psi[1], (Y psi)[1] = i psi[0] */
    const unsigned qs[1] = {q}, src[2] = {1, 0};
    const double ph[4] = {0, -1, 0, 1};
    dm_mono(s, 1, qs, src, ph, "y");
}
static void dm_h(state_t *s, qubit_t q) {
    const double u[8] = {R2, 0, R2, 0, R2, 0, -R2, 0};
    dm_mix1(s, q, u, "h");
}
static void dm_hy(state_t *s, qubit_t q) {
    /* Hy = [[1, -1], [1, 1]] / sqrt(2) */
    const double u[8] = {R2, 0, -R2, 0, R2, 0, R2, 0};
    dm_mix1(s, q, u, "hy");
}
static void dm_rx(state_t *s, qubit_t q, double theta) {
    const double c = cos(theta / 2.0), sn = sin(theta / 2.0);
    const double u[8] = {c, 0, 0, -sn, 0, -sn, c, 0};
    dm_mix1(s, q, u, "rx");
}
static void dm_ry(state_t *s, qubit_t q, double theta) {
    const double c = cos(theta / 2.0), sn = sin(theta / 2.0);
    const double u[8] = {c, 0, -sn, 0, sn, 0, c, 0};
    dm_mix1(s, q, u, "ry");
}

#define DM_BACKENDS(layout)                                                                              \
    void x_##layout(state_t *state, qubit_t target)   { dm_x(state, target); }                          \
    void y_##layout(state_t *state, qubit_t target)   { dm_y(state, target); }                          \
    void z_##layout(state_t *state, qubit_t target)   { dm_phase1(state, target, -1.0, 0.0, "z"); }     \
    void h_##layout(state_t *state, qubit_t target)   { dm_h(state, target); }                          \
    void s_##layout(state_t *state, qubit_t target)   { dm_phase1(state, target, 0.0, 1.0, "s"); }      \
    void sdg_##layout(state_t *state, qubit_t target) { dm_phase1(state, target, 0.0, -1.0, "sdg"); }   \
    void t_##layout(state_t *state, qubit_t target)   { dm_phase1(state, target, R2, R2, "t"); }        \
    void tdg_##layout(state_t *state, qubit_t target) { dm_phase1(state, target, R2, -R2, "tdg"); }     \
    void hy_##layout(state_t *state, qubit_t target)  { dm_hy(state, target); }                         \
    void rx_##layout(state_t *state, qubit_t target, double theta) { dm_rx(state, target, theta); }     \
    void ry_##layout(state_t *state, qubit_t target, double theta) { dm_ry(state, target, theta); }     \
    void rz_##layout(state_t *state, qubit_t target, double theta) {                                    \
        dm_phase1(state, target, cos(theta), sin(theta), "rz");                                         \
    }                                                                                                    \
    void p_##layout(state_t *state, qubit_t target, double theta) {                                     \
        dm_phase1(state, target, cos(theta), sin(theta), "p");                                          \
    }                                                                                                    \
    void cx_##layout(state_t *state, qubit_t control, qubit_t target) {                                 \
        const unsigned qs[2] = {control, target}, src[4] = {0, 1, 3, 2};                                \
        const double ph[8] = {1, 0, 1, 0, 1, 0, 1, 0};                                                  \
        dm_mono(state, 2, qs, src, ph, "cx");                                                           \
    }                                                                                                    \
    void cy_##layout(state_t *state, qubit_t control, qubit_t target) {                                 \
        const unsigned qs[2] = {control, target}, src[4] = {0, 1, 3, 2};                                \
        const double ph[8] = {1, 0, 1, 0, 0, -1, 0, 1};                                                 \
        dm_mono(state, 2, qs, src, ph, "cy");                                                           \
    }                                                                                                    \
    void cz_##layout(state_t *state, qubit_t control, qubit_t target) {                                 \
        const unsigned qs[2] = {control, target};                                                       \
        const double ph[8] = {1, 0, 1, 0, 1, 0, -1, 0};                                                 \
        orkan_check_cu("gate", "cz", orkan_cu_dm_phase((int)state->type, LOG_TILE_DIM, state->data,     \
                                                       state->qubits, 2, qs, ph, orkan_stream()));      \
    }                                                                                                    \
    void swap_##layout(state_t *state, qubit_t q1, qubit_t q2) {                                        \
        const unsigned qs[2] = {q1, q2}, src[4] = {0, 2, 1, 3};                                         \
        const double ph[8] = {1, 0, 1, 0, 1, 0, 1, 0};                                                  \
        dm_mono(state, 2, qs, src, ph, "swap");                                                         \
    }                                                                                                    \
    void ccx_##layout(state_t *state, qubit_t ctrl1, qubit_t ctrl2, qubit_t target) {                   \
        const unsigned qs[3] = {ctrl1, ctrl2, target}, src[8] = {0, 1, 2, 3, 4, 5, 7, 6};               \
        const double ph[16] = {1, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 0};                         \
        dm_mono(state, 3, qs, src, ph, "ccx");                                                          \
    }

DM_BACKENDS(packed)
DM_BACKENDS(tiled)

/* Arbitrary 2x2 unitary, rho -> U rho U^dagger, mat column-major (reference
 * src/gate/tiled/gate_tiled_1q.c:3-184).  Accepts both mixed layouts. */
void single_from_mat(state_t *state, qubit_t target, const cplx_t *mat) {
    GATE_VALIDATE(state && state->data && mat, "single_from_mat: null state, data or matrix pointer");
    GATE_VALIDATE(target < state->qubits, "single_from_mat: target qubit out of range");
    GATE_VALIDATE(state->type == MIXED_PACKED || state->type == MIXED_TILED,
                  "single_from_mat: mixed states only");
    double u[8];
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 2; ++c) {
            u[2 * (2 * r + c)] = creal(mat[r + 2 * c]);
            u[2 * (2 * r + c) + 1] = cimag(mat[r + 2 * c]);
        }
    dm_mix1(state, target, u, "single_from_mat");
}

/* Arbitrary 4x4 unitary on (q1, q2), mat column-major with local index
 * 2*bit(hi) + bit(lo), hi = max(q1, q2) (reference gate_tiled_2q.c:3-40). */
void two_from_mat(state_t *state, qubit_t q1, qubit_t q2, const cplx_t *mat) {
    GATE_VALIDATE(state && state->data && mat, "two_from_mat: null state, data or matrix pointer");
    GATE_VALIDATE(q1 < state->qubits && q2 < state->qubits, "two_from_mat: qubit out of range");
    GATE_VALIDATE(q1 != q2, "two_from_mat: q1 and q2 must differ");
    GATE_VALIDATE(state->type == MIXED_PACKED || state->type == MIXED_TILED, "two_from_mat: mixed states only");
    double u[32];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            u[2 * (4 * r + c)] = creal(mat[r + 4 * c]);
            u[2 * (4 * r + c) + 1] = cimag(mat[r + 4 * c]);
        }
    const unsigned qs[2] = {q1 > q2 ? q1 : q2, q1 > q2 ? q2 : q1};
    orkan_check_cu("gate", "two_from_mat",
                   orkan_cu_dm_unitary((int)state->type, LOG_TILE_DIM, state->data, state->qubits, 2, qs, u,
                                       orkan_stream()));
}

/* ---- public dispatchers ------------------------------------------------------- */
#define DISPATCH_1Q(name, state, target)                                        \
    GATE_VALIDATE((state) && (state)->data, #name ": null state or data pointer"); \
    GATE_VALIDATE((target) < (state)->qubits, #name ": target qubit out of range"); \
    switch ((state)->type) {                                                    \
        case PURE:         name##_pure(state, target);   break;                 \
        case MIXED_PACKED: name##_packed(state, target); break;                 \
        case MIXED_TILED:  name##_tiled(state, target);  break;                 \
        default: GATE_VALIDATE(0, #name ": unknown state type");                \
    }

void x(state_t *state, const qubit_t target)   { DISPATCH_1Q(x, state, target); }
void y(state_t *state, const qubit_t target)   { DISPATCH_1Q(y, state, target); }
void z(state_t *state, const qubit_t target)   { DISPATCH_1Q(z, state, target); }
void h(state_t *state, const qubit_t target)   { DISPATCH_1Q(h, state, target); }
void s(state_t *state, const qubit_t target)   { DISPATCH_1Q(s, state, target); }
void sdg(state_t *state, const qubit_t target) { DISPATCH_1Q(sdg, state, target); }
void t(state_t *state, const qubit_t target)   { DISPATCH_1Q(t, state, target); }
void tdg(state_t *state, const qubit_t target) { DISPATCH_1Q(tdg, state, target); }
void hy(state_t *state, const qubit_t target)  { DISPATCH_1Q(hy, state, target); }

#define DISPATCH_ROT(name, state, target, theta)                                \
    GATE_VALIDATE((state) && (state)->data, #name ": null state or data pointer"); \
    GATE_VALIDATE((target) < (state)->qubits, #name ": target qubit out of range"); \
    switch ((state)->type) {                                                    \
        case PURE:         name##_pure(state, target, theta);   break;          \
        case MIXED_PACKED: name##_packed(state, target, theta); break;          \
        case MIXED_TILED:  name##_tiled(state, target, theta);  break;          \
        default: GATE_VALIDATE(0, #name ": unknown state type");                \
    }

void rx(state_t *state, const qubit_t target, const double theta) { DISPATCH_ROT(rx, state, target, theta); }
void ry(state_t *state, const qubit_t target, const double theta) { DISPATCH_ROT(ry, state, target, theta); }
void rz(state_t *state, const qubit_t target, const double theta) { DISPATCH_ROT(rz, state, target, theta); }
void p(state_t *state, const qubit_t target, const double theta)  { DISPATCH_ROT(p, state, target, theta); }

#define DISPATCH_2Q(name, state, control, target)                                   \
    GATE_VALIDATE((state) && (state)->data, #name ": null state or data pointer");  \
    GATE_VALIDATE((control) < (state)->qubits, #name ": control qubit out of range"); \
    GATE_VALIDATE((target) < (state)->qubits, #name ": target qubit out of range");   \
    GATE_VALIDATE((control) != (target), #name ": control and target must differ");  \
    switch ((state)->type) {                                                        \
        case PURE:         name##_pure(state, control, target);   break;            \
        case MIXED_PACKED: name##_packed(state, control, target); break;            \
        case MIXED_TILED:  name##_tiled(state, control, target);  break;            \
        default: GATE_VALIDATE(0, #name ": unknown state type");                    \
    }

void cx(state_t *state, const qubit_t control, const qubit_t target) { DISPATCH_2Q(cx, state, control, target); }
void cy(state_t *state, const qubit_t control, const qubit_t target) { DISPATCH_2Q(cy, state, control, target); }
void cz(state_t *state, const qubit_t control, const qubit_t target) { DISPATCH_2Q(cz, state, control, target); }

void swap_gate(state_t *state, const qubit_t q1, const qubit_t q2) {
    GATE_VALIDATE(state && state->data, "swap: null state or data pointer");
    GATE_VALIDATE(q1 < state->qubits, "swap: q1 qubit out of range");
    GATE_VALIDATE(q2 < state->qubits, "swap: q2 qubit out of range");
    GATE_VALIDATE(q1 != q2, "swap: q1 and q2 must differ");
    switch (state->type) {
        case PURE:         swap_pure(state, q1, q2);   break;
        case MIXED_PACKED: swap_packed(state, q1, q2); break;
        case MIXED_TILED:  swap_tiled(state, q1, q2);  break;
        default: GATE_VALIDATE(0, "swap: unknown state type");
    }
}

void ccx(state_t *state, const qubit_t ctrl1, const qubit_t ctrl2, const qubit_t target) {
    GATE_VALIDATE(state && state->data, "ccx: null state or data pointer");
    GATE_VALIDATE(ctrl1 < state->qubits, "ccx: ctrl1 qubit out of range");
    GATE_VALIDATE(ctrl2 < state->qubits, "ccx: ctrl2 qubit out of range");
    GATE_VALIDATE(target < state->qubits, "ccx: target qubit out of range");
    GATE_VALIDATE(ctrl1 != ctrl2, "ccx: ctrl1 and ctrl2 must differ");
    GATE_VALIDATE(ctrl1 != target, "ccx: ctrl1 and target must differ");
    GATE_VALIDATE(ctrl2 != target, "ccx: ctrl2 and target must differ");
    switch (state->type) {
        case PURE:         ccx_pure(state, ctrl1, ctrl2, target);   break;
        case MIXED_PACKED: ccx_packed(state, ctrl1, ctrl2, target); break;
        case MIXED_TILED:  ccx_tiled(state, ctrl1, ctrl2, target);  break;
        default: GATE_VALIDATE(0, "ccx: unknown state type");
    }
}
