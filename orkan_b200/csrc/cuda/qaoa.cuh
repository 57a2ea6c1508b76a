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
// and each pass touches every amplitude once: a low pass works on chunks of 2^C contiguous
// amplitudes, a high pass on W = 2^(2C - n) neighbouring columns of all 2^(n - C) rows
// (x = row * 2^C + col), so the qubits it mixes are local in both.  Instances with n <= C
// run the whole circuit in one pass ("full") and never touch a state vector in memory.
//
// Inside a work item the chunk is copied into shared memory asynchronously, and the mixer
// runs in register stages of up to kQaoaGroup qubits (every thread holds 2^k amplitudes that
// differ only in the group's bits and applies the group's butterflies in registers); the
// slots of a high chunk are numbered rows first, so every group starts at slot bit 0, 4, 8
// or 12.  Rx on different qubits commute, so the order of the groups is free: the last
// stage of a pass stores from registers (or measures) with the group of the highest bits,
// so that consecutive lanes touch consecutive amplitudes of a low chunk; and segment t + 1
// starts with the group segment t ended with, so that stage applies segment t's butterflies,
// the phase between the segments and segment t + 1's butterflies without going back to
// shared memory.
//
// Arithmetic (checked against the per-call path at 1e-12): the rx pair update
// (a, b) -> (c a - i s b, c b - i s a) with c = cos(beta), s = sin(beta) (rx(2 beta) of
// gate_pure.c) is applied as k-form (a - i t b, b - i t a), t = s / c, when |c| >= |s|, or as
// (u a - i b, u b - i a), u = c / s, otherwise -- four FMAs per pair -- and the product of
// the dropped factors (c or s, once per qubit) scales each amplitude once per segment; the
// phase is (c re + s im, c im - s re) with (s, c) = sincos(cost[x] * gamma) (taken from a
// per-layer table, made by the same sincos, when the costs are stored as bytes); the mean is
// sum cost[x] |psi_x|^2 in a fixed order per chunk.
#pragma once

#include "common.cuh"

#include <math.h>

#include <type_traits>

namespace orkan {

constexpr unsigned kQaoaMaxTable = 256;   // integer costs up to 255 are stored as bytes
constexpr unsigned kQaoaGroup = 4;        // qubits per register stage
constexpr unsigned kQaoaMaxC = 13;        // 2^13 amplitudes (128 KB) staged per work item

enum QaoaKind : unsigned { kQaoaFull = 0, kQaoaLow = 1, kQaoaHigh = 2 };

struct QaoaInst {
    double2* psi;          // 2^n amplitudes (unused by full passes)
    const void* cost;      // 2^n costs: double, or uint8_t (byte costs; in high passes the
                           // transposed array of qaoa_cost_t_index)
    idx_t item0;           // first work item of this instance in the pass
    unsigned n;
    unsigned pos;          // row of the instance in the angle arrays and tables
};

// The mixer of one layer of one instance in the four-FMA form: k, which form, and the
// product of the dropped factors over the qubits a segment mixes, by pass kind
// (f[kind]: n qubits for a full pass, C for a low one, n - C for a high one).
struct QaoaRx {
    double k;
    double f[3];
    int sform;             // 0: (a - i k b) with k = s / c, scale = c; 1: (k a - i b), k = c / s, scale = s
    int pad_;
};

// Host side: the mixer coefficients of rx(theta) = exp(-i theta X / 2) from c = cos(theta / 2),
// s = sin(theta / 2), for an instance of n qubits in chunks of 2^C.
inline QaoaRx qaoa_rx_coeffs(double c, double s, unsigned n, unsigned C) {
    QaoaRx r;
    double scale;
    if (fabs(c) >= fabs(s)) { r.k = s / c; scale = c; r.sform = 0; }
    else { r.k = c / s; scale = s; r.sform = 1; }
    const unsigned nq[3] = {n, C < n ? C : n, C < n ? n - C : 0u};
    for (unsigned kd = 0; kd < 3; ++kd) {
        double f = 1.0;
        for (unsigned i = 0; i < nq[kd]; ++i) f *= scale;
        r.f[kd] = f;
    }
    r.pad_ = 0;
    return r;
}

struct QaoaTables {
    const double2* phase;  // [pos][layer][tstride]: (cos, sin)(c * gamma) for byte costs c
    const QaoaRx* rx;      // [pos][layer]
    unsigned tstride;
};

// Work items of an instance of n qubits in a pass of the given kind (low and high alike).
ORKAN_HD idx_t qaoa_items(unsigned n, unsigned C, unsigned kind) {
    return kind == kQaoaFull ? idx_t(1) : idx_t(1) << (n - C);
}
// log2 of the amplitudes of one item
ORKAN_HD unsigned qaoa_lc(unsigned n, unsigned C, unsigned kind) { return kind == kQaoaFull ? n : C; }
// log2 of the number of columns a high chunk spans
ORKAN_HD unsigned qaoa_logw(unsigned n, unsigned C) { return 2 * C - n; }

// Global amplitude index of slot s of chunk c.  Low chunk: x = c 2^C + s.  High chunk
// (rows-first): s = row + col 2^R with R = n - C row bits, x = row 2^C + c W + col.
ORKAN_HD idx_t qaoa_index(unsigned n, unsigned C, unsigned kind, idx_t c, unsigned s) {
    if (kind == kQaoaFull) return s;
    if (kind == kQaoaLow) return (c << C) + s;
    const unsigned R = n - C, lw = qaoa_logw(n, C);
    const unsigned row = s & ((1u << R) - 1), col = s >> R;
    return ((idx_t)row << C) + (c << lw) + col;
}

// Index distance of slot bit b of a mixed qubit (a row bit in high passes).
ORKAN_HD idx_t qaoa_stride(unsigned n, unsigned C, unsigned kind, unsigned b) {
    (void)n;
    return kind == kQaoaHigh ? idx_t(1) << (b + C) : idx_t(1) << b;
}

// Slot bit of qubit q.
ORKAN_HD unsigned qaoa_bit(unsigned n, unsigned C, unsigned kind, unsigned q) {
    (void)n;
    return kind == kQaoaHigh ? q - C : q;
}

// Slot of position r of a high chunk's enumeration with the K slot bits at B0 left out
// (K = 0: every slot).  Lanes 0-7 take the lowest free row bits, so the 8 lanes of a
// shared-memory phase hit consecutive slots; the next two lane bits take column bits, so a
// warp reads or writes runs of up to 4 neighbouring amplitudes (64 bytes) of 8 rows; the
// rest takes the other free row bits, then the other column bits.
ORKAN_HD unsigned qaoa_high_slot(unsigned r, unsigned R, unsigned lw, unsigned B0, unsigned K) {
    const unsigned nr = R - K;                       // free row bits
    const unsigned a = nr < 3 ? nr : 3, c = lw < 2 ? lw : 2;
    const unsigned rest = r >> (a + c);
    const unsigned rr = (r & ((1u << a) - 1)) | ((rest & ((1u << (nr - a)) - 1)) << a);
    const unsigned col = ((r >> a) & ((1u << c) - 1)) | ((rest >> (nr - a)) << c);
    const unsigned row = (rr & ((1u << B0) - 1)) | ((rr >> B0) << (B0 + K));
    return row | (col << R);
}

// Shared-memory position of slot s: one padding slot after every 16.  With the mixed qubits
// in groups of 4 slot bits starting at bit 0, 4, 8 or 12, the slots of a register set are
// then equally spaced (base + j 2^b0 sits at pad(base) + j (2^b0 + 2^(b0-4)), or + j for
// b0 = 0), and the lanes of a warp, which differ in the lowest non-group bits, fall in
// distinct banks for every group position and element size.
ORKAN_HD unsigned qaoa_pad(unsigned s) { return s + (s >> 4); }
ORKAN_HD unsigned qaoa_padded(unsigned C) { return (1u << C) + (1u << C) / 16; }

// What one pass does.
struct QaoaPlan {
    unsigned segs;             // mixer segments (1 or 2, or p for the full pass)
    unsigned q0, q1;           // qubit range of every segment
    unsigned layer0;           // layer of segment 0 (0-based); segment t is layer0 + t
    int phase_load;            // layer whose phase precedes segment 0 (-1: none)
    int init;                  // the pass starts from |+> instead of reading psi
    int measure;               // the pass ends with the mean instead of a store
    int shape;                 // group orders: 0 full (rotating), 1 first pass, 2 middle, 3 last
    unsigned m;                // register groups per segment
    unsigned nreg;             // register stages
};

ORKAN_HD QaoaPlan qaoa_plan(unsigned n, unsigned C, unsigned kind, unsigned p, unsigned j) {
    QaoaPlan pl;
    if (kind == kQaoaFull) { pl.q0 = 0; pl.q1 = n; }
    else if (kind == kQaoaLow) { pl.q0 = 0; pl.q1 = C; }
    else { pl.q0 = C; pl.q1 = n; }
    if (kind == kQaoaFull) {            // init, D1, Mix1, D2, Mix2, ..., Dp, Mixp, measure
        pl.segs = p; pl.layer0 = 0; pl.phase_load = 0; pl.init = 1; pl.measure = 1; pl.shape = 0;
    } else if (j == 0) {                // init, D1, Mix1
        pl.segs = 1; pl.layer0 = 0; pl.phase_load = 0; pl.init = 1; pl.measure = 0; pl.shape = 1;
    } else if (j < p) {                 // Mix_j, D_{j+1}, Mix_{j+1}  (0-based layers j-1, j)
        pl.segs = 2; pl.layer0 = j - 1; pl.phase_load = -1; pl.init = 0; pl.measure = 0; pl.shape = 2;
    } else {                            // Mix_p, measure
        pl.segs = 1; pl.layer0 = p - 1; pl.phase_load = -1; pl.init = 0; pl.measure = 1; pl.shape = 3;
    }
    const unsigned nq = pl.q1 - pl.q0;
    pl.m = (nq + kQaoaGroup - 1) / kQaoaGroup;
    pl.nreg = pl.m == 1 ? 1u : pl.segs * pl.m - (pl.segs - 1);
    return pl;
}

// Stages of one work item: the register stages, then two fold stages when measuring.
ORKAN_HD unsigned qaoa_stages(const QaoaPlan& pl) { return pl.nreg + (pl.measure ? 2u : 0u); }

// Group at position i of segment t's order.  Group m - 1 holds the highest slot bits; the
// first pass ends with it (store), the last starts with it (load), a middle pass does both.
ORKAN_HD unsigned qaoa_order(const QaoaPlan& pl, unsigned t, unsigned i) {
    const unsigned m = pl.m;
    switch (pl.shape) {
        case 0: return (i + m - (t % m)) % m;
        case 1: return i;
        case 3: return i == 0 ? m - 1 : i - 1;
        default:
            if (t == 0) return i == 0 ? m - 1 : i - 1;
            return i + 1 < m ? m - 2 - i : m - 1;
    }
}

enum : unsigned { kQaoaFromSmem = 0, kQaoaFromGlobal = 1, kQaoaFromInit = 2 };
enum : unsigned { kQaoaToSmem = 0, kQaoaToGlobal = 1, kQaoaToMeasure = 2 };

struct QaoaStage {
    uint8_t g;                 // group
    uint8_t t0, t1;            // segments applied in this stage
    uint8_t src, dst;
    int8_t pre_phase;          // phase of segment t0's preceding layer applied before it (-1: none)
    uint8_t end0;              // segment t0 ends in this stage (all of t0..t1 when there is one group)
    uint8_t pad_;
};

// Register stage r of a pass.  Stages 0..m-1 run segment 0's groups; every later segment
// adds m - 1 stages (its first group shares the previous segment's last stage).
ORKAN_HD QaoaStage qaoa_reg_stage(const QaoaPlan& pl, unsigned r) {
    QaoaStage s;
    s.pad_ = 0;
    if (pl.m == 1) {
        s.g = 0; s.t0 = 0; s.t1 = (uint8_t)(pl.segs - 1); s.end0 = 1;
    } else {
        unsigned t, i;
        if (r < pl.m) { t = 0; i = r; }
        else { const unsigned k = r - pl.m; t = 1 + k / (pl.m - 1); i = 1 + k % (pl.m - 1); }
        s.g = (uint8_t)qaoa_order(pl, t, i);
        s.t0 = (uint8_t)t;
        s.t1 = (uint8_t)((i == pl.m - 1 && t + 1 < pl.segs) ? t + 1 : t);
        s.end0 = i == pl.m - 1;
    }
    s.src = (r == 0 && pl.init) ? kQaoaFromInit : kQaoaFromSmem;
    s.dst = r + 1 == pl.nreg ? (pl.measure ? kQaoaToMeasure : kQaoaToGlobal) : kQaoaToSmem;
    s.pre_phase = (int8_t)((r == 0) ? pl.phase_load : -1);
    return s;
}

// A pass launch: its instances (all of one qubit count), the pass's plan and, when they
// fit, its register stages, computed once on the host.
constexpr unsigned kQaoaStageTable = 16;

struct QaoaPass {
    const QaoaInst* inst;
    unsigned ninst;
    idx_t items;           // total work items of the pass
    const double* gamma;   // [pos][p]
    double* partial;       // measuring pass: one partial sum per work item
    unsigned p;
    unsigned pass;         // j in [0, p] (0 for full passes)
    unsigned C;            // log2 of the chunk (amplitudes per item)
    unsigned kind;         // QaoaKind
    QaoaPlan plan;         // qaoa_plan(n, C, kind, p, pass) of the launch's qubit count
    unsigned li;           // log2 of the work items per instance: item w is chunk w mod 2^li
                           // of instance w >> li of the list (every instance has n qubits)
    int table_layer;       // the layer of the pass's one phase (low and high passes), whose
                           // table byte-cost launches stage in shared memory; -1: none
    QaoaStage stage[kQaoaStageTable];   // qaoa_reg_stage(plan, r) for r < nreg <= kQaoaStageTable
};

// Fill in the plan and the stage table of a pass of n-qubit instances.
ORKAN_HD void qaoa_pass_setup(QaoaPass& P, unsigned n) {
    P.plan = qaoa_plan(n, P.C, P.kind, P.p, P.pass);
    P.li = P.kind == kQaoaFull ? 0u : n - P.C;
    P.table_layer = P.kind == kQaoaFull ? -1
                    : P.plan.phase_load >= 0 ? (int)P.plan.layer0 + P.plan.phase_load
                    : P.plan.segs > 1 ? (int)P.plan.layer0 + 1 : -1;
    for (unsigned r = 0; r < kQaoaStageTable; ++r)
        P.stage[r] = r < P.plan.nreg ? qaoa_reg_stage(P.plan, r) : QaoaStage{};
}
ORKAN_HD QaoaStage qaoa_stage_desc(const QaoaPass& P, unsigned r) {
    return P.plan.nreg <= kQaoaStageTable ? P.stage[r] : qaoa_reg_stage(P.plan, r);
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

// Shared memory of one block: kQaoaRing buffers, each vb[2^C] amplitudes (padded), the
// phase table (byte costs) and the costs: FP64 costs one per padded slot (cw), byte costs
// as a byte array cb copied in 16-byte runs (see qaoa_cost_index); then red[nthr + 32].
constexpr unsigned kQaoaRing = 2;

template <class CostT>
struct QaoaSmem {
    double2* vb;
    double* cw;            // FP64 costs: one per padded slot
    uint8_t* cb;           // byte costs (qaoa_cost_index layout)
    double2* tab;          // byte costs: the staged phase table of the pass's phase layer
    double* red;
};

// Byte costs of high passes come from the instance's transposed cost array,
// cost_t[col 2^R + row] = cost[row 2^C + col] (R = n - C), so that a high chunk's costs, the
// W columns chunk W .. chunk W + W - 1 of every row in slot order (s = row + col 2^R), are
// the contiguous run cost_t[chunk 2^C .. chunk 2^C + 2^C) and copy in 16-byte pieces like a
// low chunk's (instead of a 1-4 byte word from each of 2^R rows 2^C bytes apart).
ORKAN_HD idx_t qaoa_cost_t_index(unsigned n, unsigned C, idx_t x) {
    const unsigned R = n - C;
    return ((x & ((idx_t(1) << C) - 1)) << R) | (x >> C);
}

// Position of slot s's byte cost in cb: s, the chunk's costs being contiguous (low and full
// chunks in the cost array, high chunks in the transposed one); chunks of fewer than 4
// costs copy the aligned 4-byte word holding them, so their costs start at byte
// (chunk 2^C) mod 4.
ORKAN_HD unsigned qaoa_cost_index(unsigned kind, unsigned C, idx_t chunk, unsigned s) {
    if (kind == kQaoaFull) return s;
    return C >= 2 ? s : (unsigned)((chunk << C) & 3u) + s;
}

// Bytes of the byte-cost array of a chunk of 2^C amplitudes, at least 16 for the 16-byte
// copies of tiny full chunks.
ORKAN_HD size_t qaoa_cost_bytes(unsigned C) { return C < 4 ? 16u : (size_t(1) << C); }

// Phase-table entries a buffer holds: kQaoaMaxTable for byte costs, none for FP64 costs.
template <class CostT>
ORKAN_HD constexpr unsigned qaoa_table_slots() { return std::is_same<CostT, double>::value ? 0u : kQaoaMaxTable; }

// Bytes of one buffer, rounded up to 128 so that every buffer, its costs and the reduction
// array after the last buffer keep the alignment of the shared-memory base.
template <class CostT>
ORKAN_HD size_t qaoa_buffer_bytes(unsigned C) {
    const size_t cost = std::is_same<CostT, double>::value ? size_t(8) * qaoa_padded(C) : qaoa_cost_bytes(C);
    const size_t b = size_t(16) * qaoa_padded(C) + size_t(16) * qaoa_table_slots<CostT>() + cost;
    return (b + 127) & ~size_t(127);
}

// Alignment of every region of a block's shared memory (base aligned to 128 bytes): the
// 16-byte amplitudes and the asynchronous copies into them, the costs (16-byte copies of
// byte runs), the doubles of the reduction.
template <class CostT>
ORKAN_HD bool qaoa_smem_aligned(unsigned C, unsigned ring) {
    for (unsigned slot = 0; slot < ring; ++slot) {
        const size_t vb = qaoa_buffer_bytes<CostT>(C) * slot, tab = vb + size_t(16) * qaoa_padded(C);
        const size_t cost = tab + size_t(16) * qaoa_table_slots<CostT>();
        if (vb % 16 || tab % 16 || cost % 16) return false;
    }
    return (qaoa_buffer_bytes<CostT>(C) * ring) % 8 == 0;
}
template <class CostT>
ORKAN_HD size_t qaoa_smem_bytes(unsigned C, unsigned nthr, unsigned ring) {
    return qaoa_buffer_bytes<CostT>(C) * ring + size_t(8) * (nthr + 32);
}
template <class CostT>
ORKAN_HD QaoaSmem<CostT> qaoa_smem_at(unsigned char* base, unsigned C, unsigned nthr, unsigned ring, unsigned slot) {
    QaoaSmem<CostT> S;
    unsigned char* b = base + qaoa_buffer_bytes<CostT>(C) * slot;
    S.vb = reinterpret_cast<double2*>(b);
    // [amplitudes, 16 B each][phase table, 16 B each][costs]: every region aligned
    S.tab = qaoa_table_slots<CostT>() ? reinterpret_cast<double2*>(b + size_t(16) * qaoa_padded(C)) : nullptr;
    unsigned char* c = b + size_t(16) * (qaoa_padded(C) + qaoa_table_slots<CostT>());
    S.cw = std::is_same<CostT, double>::value ? reinterpret_cast<double*>(c) : nullptr;
    S.cb = std::is_same<CostT, double>::value ? nullptr : reinterpret_cast<uint8_t*>(c);
    S.red = reinterpret_cast<double*>(base + qaoa_buffer_bytes<CostT>(C) * ring);
    (void)nthr;
    return S;
}

// Fill of one work item's buffer: asynchronous copies of its amplitudes (unless the pass
// starts from |+>), slot s = tid, tid + nthr, ... in order, so consecutive threads copy
// consecutive amplitudes, and of its costs: FP64 costs per slot, byte costs as one
// contiguous run in 16-byte copies (I.cost is the transposed array in high passes).
// Mem::cp16(dst, x) copies amplitude x; CostMem::cpw(dst, x) the FP64 cost of amplitude
// x; CostMem::cpb(dst, x, bytes) bytes byte costs from amplitude x (x a multiple of bytes).
template <class CostT, class Mem, class CostMem>
ORKAN_HD void qaoa_fill(const QaoaPass& P, const QaoaTables& T, const QaoaInst& I, const QaoaPlan& pl, const Mem& psi,
                        const CostMem& cost, idx_t chunk, const QaoaSmem<CostT>& S, unsigned tid, unsigned nthr) {
    const unsigned cnt = 1u << qaoa_lc(I.n, P.C, P.kind);
    if (qaoa_table_slots<CostT>() && P.table_layer >= 0) {    // the phase table of the pass
        const double2* row = T.phase + ((idx_t)I.pos * P.p + (unsigned)P.table_layer) * T.tstride;
        for (unsigned e = tid; e < T.tstride; e += nthr) psi.cpg(S.tab + e, row + e);
    }
    constexpr bool kBytes = !std::is_same<CostT, double>::value;
    if (P.kind != kQaoaHigh) {                     // contiguous chunk: equally spaced copies
        const idx_t x0 = P.kind == kQaoaLow ? chunk << P.C : 0;
        for (unsigned e = tid; e < cnt; e += nthr) {
            if (!pl.init) psi.cp16(S.vb + qaoa_pad(e), x0 + e);
            if constexpr (!kBytes) cost.cpw(S.cw + qaoa_pad(e), x0 + e);
        }
    } else {
        const unsigned R = I.n - P.C, lw = qaoa_logw(I.n, P.C);
        for (unsigned e = tid; e < cnt; e += nthr) {
            const unsigned s = qaoa_high_slot(e, R, lw, 0, 0);
            const idx_t x = qaoa_index(I.n, P.C, P.kind, chunk, s);
            if (!pl.init) psi.cp16(S.vb + qaoa_pad(s), x);
            if constexpr (!kBytes) cost.cpw(S.cw + qaoa_pad(s), x);
        }
    }
    if constexpr (kBytes) {                        // one contiguous run (transposed in high passes)
        const idx_t x0 = P.kind == kQaoaFull ? 0 : chunk << P.C;
        if (cnt >= 16 || P.kind == kQaoaFull) {   // 16 costs per copy (whole 16-byte units)
            for (unsigned e = 16 * tid; e < cnt || (e == 0 && cnt < 16); e += 16 * nthr)
                cost.cpb(S.cb + e, x0 + e, 16);
        } else if (tid == 0) {                    // a chunk of 1-8 costs: one copy
            if (cnt >= 4) cost.cpb(S.cb, x0, cnt);
            else cost.cpb(S.cb, x0 & ~idx_t(3), 4);
        }
    }
}

// Register stage of a group of K slot bits starting at B0 (0, 4, 8 or 12).
template <int K, int B0, class CostT, class Mem>
ORKAN_HD void qaoa_group(const QaoaPass& P, const QaoaTables& T, const QaoaInst& I, const QaoaPlan& pl,
                         const QaoaStage& sg, const Mem& psi, idx_t chunk, const QaoaSmem<CostT>& S, unsigned lc,
                         unsigned tid, unsigned nthr) {
    constexpr unsigned NV = 1u << K;
    constexpr unsigned D = B0 == 0 ? 1u : (1u << B0) + (1u << (B0 - 4));   // padded distance of element j
    constexpr unsigned LOWM = (1u << B0) - 1;
    const unsigned n = I.n;
    const unsigned sets = 1u << (lc - K);
    const idx_t xs = qaoa_stride(n, P.C, P.kind, B0);
    const idx_t row = (idx_t)I.pos * P.p;
    const double amp0 = 1.0 / sqrt((double)(idx_t(1) << n));
    double acc = 0.0;
    const bool high = P.kind == kQaoaHigh;
    const unsigned R = high ? n - P.C : 0u, lw = high ? qaoa_logw(n, P.C) : 0u;
    for (unsigned r = tid; r < sets; r += nthr) {
        const unsigned base = high ? qaoa_high_slot(r, R, lw, B0, K) : (r & LOWM) | ((r >> B0) << (B0 + K));
        const unsigned p0 = qaoa_pad(base);
        const idx_t xb = qaoa_index(n, P.C, P.kind, chunk, base);      // slot base | j << B0 is xb + j xs
        // cost of element j, read from the staged costs where it is used
        auto cost_of = [&](unsigned j) -> CostT {
            if constexpr (std::is_same<CostT, double>::value) {
                return S.cw[p0 + j * D];
            } else {
                return S.cb[qaoa_cost_index(P.kind, P.C, chunk, base | (j << B0))];
            }
        };
        double2 v[NV];
        if (sg.src == kQaoaFromSmem) {
#pragma unroll
            for (unsigned j = 0; j < NV; ++j) v[j] = S.vb[p0 + j * D];
        } else {
#pragma unroll
            for (unsigned j = 0; j < NV; ++j) v[j] = c2(amp0, 0.0);
        }
        if (sg.pre_phase >= 0) {
            const unsigned layer = pl.layer0 + (unsigned)sg.pre_phase;
            const double gam = P.gamma[row + layer];
            const double2* tb = (int)layer == P.table_layer && S.tab ? S.tab : T.phase + (row + layer) * T.tstride;
#pragma unroll
            for (unsigned j = 0; j < NV; ++j) v[j] = qaoa_apply_phase(qaoa_phase<CostT>(cost_of(j), gam, tb), v[j]);
        }
        for (unsigned t = sg.t0; t <= sg.t1; ++t) {
            const unsigned layer = pl.layer0 + t;
            const QaoaRx& rx = T.rx[row + layer];
            const double k = rx.k;
            if (rx.sform == 0) {
#pragma unroll
                for (unsigned b = 0; b < (unsigned)K; ++b)
#pragma unroll
                    for (unsigned j = 0; j < NV; ++j)
                        if (!(j & (1u << b))) {
                            double2& a = v[j];
                            double2& c = v[j | (1u << b)];
                            const double2 na = c2(fma(k, c.y, a.x), fma(-k, c.x, a.y));
                            c = c2(fma(k, a.y, c.x), fma(-k, a.x, c.y));
                            a = na;
                        }
            } else {
#pragma unroll
                for (unsigned b = 0; b < (unsigned)K; ++b)
#pragma unroll
                    for (unsigned j = 0; j < NV; ++j)
                        if (!(j & (1u << b))) {
                            double2& a = v[j];
                            double2& c = v[j | (1u << b)];
                            const double2 na = c2(fma(k, a.x, c.y), fma(k, a.y, -c.x));
                            c = c2(fma(k, c.x, a.y), fma(k, c.y, -a.x));
                            a = na;
                        }
            }
            const bool ends = (pl.m == 1) || (t == sg.t0 && sg.end0);
            if (t < sg.t1) {                                  // scale of segment t, phase of the next layer
                const double f = rx.f[P.kind];
                const double gam = P.gamma[row + layer + 1];
                const double2* tb = (int)layer + 1 == P.table_layer && S.tab ? S.tab
                                                                             : T.phase + (row + layer + 1) * T.tstride;
#pragma unroll
                for (unsigned j = 0; j < NV; ++j) {
                    const double2 ph = qaoa_phase<CostT>(cost_of(j), gam, tb);
                    v[j] = qaoa_apply_phase(c2(ph.x * f, ph.y * f), v[j]);
                }
            } else if (ends) {
                const double f = rx.f[P.kind];
#pragma unroll
                for (unsigned j = 0; j < NV; ++j) v[j] = c2(v[j].x * f, v[j].y * f);
            }
        }
        if (sg.dst == kQaoaToMeasure) {
#pragma unroll
            for (unsigned j = 0; j < NV; ++j) acc += (double)cost_of(j) * (v[j].x * v[j].x + v[j].y * v[j].y);
        } else if (sg.dst == kQaoaToGlobal) {
#pragma unroll
            for (unsigned j = 0; j < NV; ++j) psi.st(xb + j * xs, v[j]);
        } else {
#pragma unroll
            for (unsigned j = 0; j < NV; ++j) S.vb[p0 + j * D] = v[j];
        }
    }
    if (sg.dst == kQaoaToMeasure) S.red[tid] = acc;
}

// Per-thread work of stage `st` of one work item (instance I, chunk index `chunk`) whose
// buffer S was filled by qaoa_fill.  Barriers between the stages are the caller's.
template <class CostT, class Mem>
ORKAN_HD void qaoa_stage(const QaoaPass& P, const QaoaTables& T, const QaoaInst& I, const QaoaPlan& pl,
                         const Mem& psi, idx_t chunk, unsigned st, const QaoaSmem<CostT>& S, unsigned tid,
                         unsigned nthr) {
    const unsigned n = I.n, kind = P.kind;
    if (st < pl.nreg) {
        const QaoaStage sg = qaoa_stage_desc(P, st);
        const unsigned lc = qaoa_lc(n, P.C, kind);
        const unsigned nq = pl.q1 - pl.q0;
        const unsigned off = sg.g * kQaoaGroup;
        const unsigned k = (nq - off) < kQaoaGroup ? nq - off : kQaoaGroup;
        const unsigned b0 = qaoa_bit(n, P.C, kind, pl.q0 + off);     // 0, 4, 8 or 12
#define ORKAN_QAOA_GROUP(KK, BB) \
    case (KK) * 16 + (BB): qaoa_group<KK, BB, CostT>(P, T, I, pl, sg, psi, chunk, S, lc, tid, nthr); break;
        switch (k * 16 + b0) {
            ORKAN_QAOA_GROUP(1, 0) ORKAN_QAOA_GROUP(2, 0) ORKAN_QAOA_GROUP(3, 0) ORKAN_QAOA_GROUP(4, 0)
            ORKAN_QAOA_GROUP(1, 4) ORKAN_QAOA_GROUP(2, 4) ORKAN_QAOA_GROUP(3, 4) ORKAN_QAOA_GROUP(4, 4)
            ORKAN_QAOA_GROUP(1, 8) ORKAN_QAOA_GROUP(2, 8) ORKAN_QAOA_GROUP(3, 8) ORKAN_QAOA_GROUP(4, 8)
            ORKAN_QAOA_GROUP(1, 12) ORKAN_QAOA_GROUP(2, 12) ORKAN_QAOA_GROUP(3, 12) ORKAN_QAOA_GROUP(4, 12)
            default: break;
        }
#undef ORKAN_QAOA_GROUP
        return;
    }
    // fold of the per-thread sums in a fixed order: 32 strided partial sums, then one
    if (st == pl.nreg) {
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

#ifdef __CUDACC__
// Device accessors: amplitude loads/stores and the asynchronous 16-byte copy of the fill.
struct QaoaDevPsi {
    double2* p;
    __device__ __forceinline__ void st(idx_t i, double2 v) const { p[i] = v; }
    __device__ __forceinline__ void cp16(double2* dst, idx_t i) const {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(p + i) : "memory");
    }
    __device__ __forceinline__ void cpg(double2* dst, const double2* src) const {   // a table entry
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
    }
};
template <class CostT>
struct QaoaDevCost;
template <>
struct QaoaDevCost<double> {
    const double* p;
    __device__ __forceinline__ void cpw(double* dst, idx_t i) const {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(p + i) : "memory");
    }
};
template <>
struct QaoaDevCost<uint8_t> {
    const uint8_t* p;            // allocated in whole 16-byte units
    // `bytes` (4, 8 or 16) costs from amplitude i (a multiple of bytes) to dst
    __device__ __forceinline__ void cpb(uint8_t* dst, idx_t i, unsigned bytes) const {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
        if (bytes == 16)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(p + i) : "memory");
        else if (bytes == 8)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(p + i) : "memory");
        else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(p + i) : "memory");
    }
};
__device__ __forceinline__ void qaoa_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void qaoa_cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
#endif

}  // namespace orkan
