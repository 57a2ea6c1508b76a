// qaoa.cuh - batched QAOA-style circuits of uneven sizes, fused into p + 1 passes.
//
// Each instance (n qubits, diagonal cost vector cost, angles gamma_k, beta_k) is the
// composition of the reference's own calls (no reference counterpart as a whole):
//     state_plus(n)                                     src/state/state_pure.c:30-43
//     for k < p:  exp_diag(cost, gamma_k)               src/circ/circ_pure.c:21-33
//                 rx(q, 2 beta_k) for every qubit q     src/gate/gate_pure.c:230-234
//     mean(cost)                                        src/meas/meas_pure.c:20-30
// The mixer of layer k factors into L_k (rx on qubits < C) and H_k (rx on qubits >= C),
// which commute, so the circuit D1 L1 H1 D2 L2 H2 ... Dp Lp Hp M regroups as
//     pass 0 (low):           init, D1, L1
//     pass j (1 <= j < p):    Mix_j, D_{j+1}, Mix_{j+1}   with Mix = H (j odd) or L (j even)
//     pass p:                 Mix_p, M
// and each pass touches every amplitude once: a low pass stages 2^C contiguous amplitudes,
// a high pass stages W = 2^(2C - n) neighbouring columns of all 2^(n - C) rows (x = row *
// 2^C + col), so the qubits it mixes are local in both.  Instances with n <= C run the
// whole circuit in one pass ("full") and never touch a state vector in device memory.
//
// Inside a work item the staged chunk lives in shared memory; the mixer runs in register
// stages of up to kQaoaGroup qubits each (every thread holds 2^k amplitudes that differ
// only in the group's bits and applies the group's butterflies in registers).  Rx on
// different qubits commute, so segment t + 1 starts with the group segment t ended with;
// that stage applies segment t's butterflies, the phase between the segments and
// segment t + 1's butterflies without going back to shared memory.
//
// Arithmetic matches the per-call path: rx uses the pair formula of gate_pure.c with
// c = cos(beta), s = sin(beta) (rx(2 beta) takes cos(2 beta / 2), the same value); the
// phase is (c re + s im, c im - s re) with (s, c) = sincos(cost[x] * gamma) (taken from a
// per-layer table, made by the same sincos, when the costs are stored as bytes); the mean
// is sum cost[x] |psi_x|^2, in a fixed order per chunk.
#pragma once

#include "common.cuh"
#include "pure.cuh"

#include <type_traits>

namespace orkan {

constexpr unsigned kQaoaMaxTable = 256;   // integer costs up to 255 are stored as bytes
constexpr unsigned kQaoaGroup = 4;        // qubits per register stage
constexpr unsigned kQaoaMaxC = 13;        // 2^13 amplitudes (128 KB) staged per work item

enum QaoaKind : unsigned { kQaoaFull = 0, kQaoaLow = 1, kQaoaHigh = 2 };

struct QaoaInst {
    double2* psi;          // 2^n amplitudes (unused by full passes)
    const void* cost;      // 2^n costs: double, or uint8_t (byte costs)
    idx_t item0;           // first work item of this instance in the pass
    unsigned n;
    unsigned pos;          // row of the instance in the angle arrays and tables
};

struct QaoaPass {
    const QaoaInst* inst;
    unsigned ninst;
    idx_t items;           // total work items of the pass
    const double* gamma;   // [pos][p]
    double* partial;       // measuring pass: one partial sum per work item
    unsigned p;
    unsigned pass;         // j in [0, p] (0 for full passes)
    unsigned C;            // log2 of the chunk (amplitudes staged per item)
    unsigned kind;         // QaoaKind
};

struct QaoaTables {
    const double2* phase;  // [pos][layer][tstride]: (cos, sin)(c * gamma) for byte costs c
    const double2* rx;     // [pos][layer]: (cos(beta), sin(beta)) as the host computes them
    unsigned tstride;
};

// Work items of an instance of n qubits in a pass of the given kind (low and high alike).
ORKAN_HD idx_t qaoa_items(unsigned n, unsigned C, unsigned kind) {
    return kind == kQaoaFull ? idx_t(1) : idx_t(1) << (n - C);
}
// log2 of the staged amplitudes of one item
ORKAN_HD unsigned qaoa_lc(unsigned n, unsigned C, unsigned kind) { return kind == kQaoaFull ? n : C; }
// log2 of the number of columns a high chunk spans
ORKAN_HD unsigned qaoa_logw(unsigned n, unsigned C) { return 2 * C - n; }

// Global amplitude index of staged slot s of chunk c.
ORKAN_HD idx_t qaoa_index(unsigned n, unsigned C, unsigned kind, idx_t c, unsigned s) {
    if (kind == kQaoaFull) return s;
    if (kind == kQaoaLow) return (c << C) + s;
    const unsigned lw = qaoa_logw(n, C);
    const unsigned row = s >> lw, col = s & ((1u << lw) - 1);
    return ((idx_t)row << C) + (c << lw) + col;
}

// Staged-slot bit of qubit q.
ORKAN_HD unsigned qaoa_bit(unsigned n, unsigned C, unsigned kind, unsigned q) {
    return kind == kQaoaHigh ? q - C + qaoa_logw(n, C) : q;
}

// Work item w -> position in the pass's instance list (binary search over item0).
ORKAN_HD unsigned qaoa_find(const QaoaInst* inst, unsigned ninst, idx_t w) {
    unsigned lo = 0, hi = ninst;
    while (hi - lo > 1) {
        const unsigned mid = (lo + hi) >> 1;
        if (inst[mid].item0 <= w) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Shared-memory slot permutations that keep the register stages free of bank conflicts
// for every group position (16-byte amplitudes, 8- and 1-byte costs).
ORKAN_HD unsigned qaoa_sw16(unsigned s) { return s ^ ((s >> 4) & 7u); }
ORKAN_HD unsigned qaoa_sw8(unsigned s) { return s ^ ((s >> 4) & 15u); }

// What one pass does.
struct QaoaPlan {
    unsigned segs;             // mixer segments (1 or 2, or p for the full pass)
    unsigned q0, q1;           // qubit range of every segment
    unsigned layer0;           // layer of segment 0 (0-based); segment t is layer0 + t
    int phase_load;            // layer whose phase follows the load (-1: none)
    int init;                  // the load stage generates |+> instead of reading psi
    int measure;               // the pass ends with the mean instead of a store
    unsigned m;                // register groups per segment
    unsigned nreg;             // register stages
};

ORKAN_HD QaoaPlan qaoa_plan(unsigned n, unsigned C, unsigned kind, unsigned p, unsigned j) {
    QaoaPlan pl;
    if (kind == kQaoaFull) { pl.q0 = 0; pl.q1 = n; }
    else if (kind == kQaoaLow) { pl.q0 = 0; pl.q1 = C; }
    else { pl.q0 = C; pl.q1 = n; }
    if (kind == kQaoaFull) {            // init, D1, Mix1, D2, Mix2, ..., Dp, Mixp, measure
        pl.segs = p; pl.layer0 = 0; pl.phase_load = 0; pl.init = 1; pl.measure = 1;
    } else if (j == 0) {                // init, D1, Mix1
        pl.segs = 1; pl.layer0 = 0; pl.phase_load = 0; pl.init = 1; pl.measure = 0;
    } else if (j < p) {                 // Mix_j, D_{j+1}, Mix_{j+1}  (0-based layers j-1, j)
        pl.segs = 2; pl.layer0 = j - 1; pl.phase_load = -1; pl.init = 0; pl.measure = 0;
    } else {                            // Mix_p, measure
        pl.segs = 1; pl.layer0 = p - 1; pl.phase_load = -1; pl.init = 0; pl.measure = 1;
    }
    const unsigned nq = pl.q1 - pl.q0;
    pl.m = (nq + kQaoaGroup - 1) / kQaoaGroup;
    pl.nreg = pl.m == 1 ? 1u : pl.segs * pl.m - (pl.segs - 1);
    return pl;
}

// Stages of one work item: load, the register stages, then store (or two fold stages).
ORKAN_HD unsigned qaoa_stages(const QaoaPlan& pl) { return 1 + pl.nreg + (pl.measure ? 2u : 1u); }

// Register stage r: group g, applied for segments t0..t1 (t1 = t0 + 1 when the stage
// carries the phase between two segments; all segments when there is a single group).
ORKAN_HD void qaoa_reg_stage(const QaoaPlan& pl, unsigned r, unsigned* g, unsigned* t0, unsigned* t1) {
    if (pl.m == 1) { *g = 0; *t0 = 0; *t1 = pl.segs - 1; return; }
    unsigned t, i;
    if (r < pl.m) { t = 0; i = r; }
    else { const unsigned k = r - pl.m; t = 1 + k / (pl.m - 1); i = 1 + k % (pl.m - 1); }
    *g = (i + pl.m - (t % pl.m)) % pl.m;
    *t0 = t;
    *t1 = (i == pl.m - 1 && t + 1 < pl.segs) ? t + 1 : t;
}

ORKAN_HD double2 qaoa_apply_phase(double2 ph, double2 v) {
    return c2(ph.x * v.x + ph.y * v.y, ph.x * v.y - ph.y * v.x);
}

template <class CostT>
ORKAN_HD double2 qaoa_phase(CostT c, double gamma, const double2* table) {
    if constexpr (std::is_same<CostT, double>::value) {
        (void)table;
        double sn, cs;
        sincos(c * gamma, &sn, &cs);
        return c2(cs, sn);
    } else {
        (void)gamma;
        return table[c];
    }
}

// Shared memory of one block: vb[2^C] amplitudes, red[nthr + 32] doubles, cb[2^C] costs.
template <class CostT>
struct QaoaSmem {
    double2* vb;
    double* red;
    CostT* cb;
};

template <class CostT>
ORKAN_HD size_t qaoa_smem_bytes(unsigned C, unsigned nthr) {
    return (size_t(16) + sizeof(CostT)) * (size_t(1) << C) + size_t(8) * (nthr + 32);
}

// Register stage of a group of K slot bits starting at b0.
template <int K, class CostT>
ORKAN_HD void qaoa_group(const QaoaPass& P, const QaoaTables& T, const QaoaInst& I, const QaoaPlan& pl,
                         const QaoaSmem<CostT>& S, unsigned lc, unsigned b0, unsigned t0, unsigned t1,
                         bool measure, unsigned tid, unsigned nthr) {
    constexpr unsigned NV = 1u << K;
    const unsigned sets = 1u << (lc - K);
    const unsigned lowm = (1u << b0) - 1;
    double acc = 0.0;
    for (unsigned r = tid; r < sets; r += nthr) {
        const unsigned base = (r & lowm) | ((r >> b0) << (b0 + K));
        double2 v[NV];
#pragma unroll
        for (unsigned j = 0; j < NV; ++j) v[j] = S.vb[qaoa_sw16(base | (j << b0))];
        for (unsigned t = t0; t <= t1; ++t) {
            const unsigned layer = pl.layer0 + t;
            const double2 cs = T.rx[(idx_t)I.pos * P.p + layer];
#pragma unroll
            for (unsigned b = 0; b < (unsigned)K; ++b) {
#pragma unroll
                for (unsigned j = 0; j < NV; ++j)
                    if (!(j & (1u << b))) pair_op<kOpRx>(v[j], v[j | (1u << b)], cs.x, cs.y);
            }
            if (t < t1) {                                     // phase of the next layer
                const double gam = P.gamma[(idx_t)I.pos * P.p + layer + 1];
                const double2* tb = T.phase + ((idx_t)I.pos * P.p + layer + 1) * T.tstride;
#pragma unroll
                for (unsigned j = 0; j < NV; ++j)
                    v[j] = qaoa_apply_phase(qaoa_phase<CostT>(S.cb[qaoa_sw8(base | (j << b0))], gam, tb), v[j]);
            }
        }
        if (measure) {
#pragma unroll
            for (unsigned j = 0; j < NV; ++j)
                acc += (double)S.cb[qaoa_sw8(base | (j << b0))] * (v[j].x * v[j].x + v[j].y * v[j].y);
        } else {
#pragma unroll
            for (unsigned j = 0; j < NV; ++j) S.vb[qaoa_sw16(base | (j << b0))] = v[j];
        }
    }
    if (measure) S.red[tid] = acc;
}

// Per-thread work of stage `st` of one work item (instance I, chunk index `chunk`).
// Barriers between the stages are the caller's.
template <class CostT, class Mem, class CostMem>
ORKAN_HD void qaoa_stage(const QaoaPass& P, const QaoaTables& T, const QaoaInst& I, const QaoaPlan& pl,
                         const Mem& psi, const CostMem& cost, idx_t chunk, unsigned st, const QaoaSmem<CostT>& S,
                         unsigned tid, unsigned nthr) {
    const unsigned n = I.n, kind = P.kind;
    const unsigned lc = qaoa_lc(n, P.C, kind);
    const unsigned cnt = 1u << lc;
    if (st == 0) {                                            // load (or |+>), costs, the load phase
        const double amp = 1.0 / sqrt((double)(idx_t(1) << n));
        const double gam = pl.phase_load >= 0 ? P.gamma[(idx_t)I.pos * P.p + (unsigned)pl.phase_load] : 0.0;
        const double2* tb = T.phase + ((idx_t)I.pos * P.p + (pl.phase_load >= 0 ? pl.phase_load : 0)) * T.tstride;
        for (unsigned s = tid; s < cnt; s += nthr) {
            const idx_t x = qaoa_index(n, P.C, kind, chunk, s);
            const CostT c = cost.ld(x);
            double2 v = pl.init ? c2(amp, 0.0) : psi.ld(x);
            if (pl.phase_load >= 0) v = qaoa_apply_phase(qaoa_phase<CostT>(c, gam, tb), v);
            S.cb[qaoa_sw8(s)] = c;
            S.vb[qaoa_sw16(s)] = v;
        }
        return;
    }
    if (st <= pl.nreg) {                                      // one register stage
        unsigned g, t0, t1;
        qaoa_reg_stage(pl, st - 1, &g, &t0, &t1);
        const unsigned nq = pl.q1 - pl.q0;
        const unsigned off = g * kQaoaGroup;
        const unsigned k = (nq - off) < kQaoaGroup ? nq - off : kQaoaGroup;
        const unsigned b0 = qaoa_bit(n, P.C, kind, pl.q0 + off);
        const bool measure = pl.measure && st == pl.nreg;
        switch (k) {
            case 1: qaoa_group<1>(P, T, I, pl, S, lc, b0, t0, t1, measure, tid, nthr); break;
            case 2: qaoa_group<2>(P, T, I, pl, S, lc, b0, t0, t1, measure, tid, nthr); break;
            case 3: qaoa_group<3>(P, T, I, pl, S, lc, b0, t0, t1, measure, tid, nthr); break;
            default: qaoa_group<4>(P, T, I, pl, S, lc, b0, t0, t1, measure, tid, nthr); break;
        }
        return;
    }
    if (!pl.measure) {                                        // store
        for (unsigned s = tid; s < cnt; s += nthr) psi.st(qaoa_index(n, P.C, kind, chunk, s), S.vb[qaoa_sw16(s)]);
        return;
    }
    // fold of the per-thread sums in a fixed order: 32 strided partial sums, then one
    if (st == pl.nreg + 1) {
        if (tid < 32) {
            double s = 0.0;
            for (unsigned t = tid; t < nthr; t += 32) s += S.red[t];
            S.red[nthr + tid] = s;
        }
    } else if (tid == 0) {
        double s = 0.0;
        for (unsigned t = 0; t < 32; ++t) s += S.red[nthr + t];
        P.partial[I.item0 + chunk] = s;
    }
}

}  // namespace orkan
