// emu.cpp - CPU emulation of the CUDA kernels' index logic -- TEST INFRASTRUCTURE ONLY.
//
// The kernels in orkan_b200/csrc/cuda are written as __host__ __device__ per-thread
// (and per-phase) functions over a memory accessor.  This file instantiates the same
// functions with a checking accessor and runs every thread of every block on the CPU,
// with block barriers honoured by running each phase for all threads before the next.
// The accessor rejects out-of-range indices and counts reads and writes per element, so
// the tests can prove, before any GPU run, that every access of a launch stays inside
// the storage and that each stored element is read and written exactly as often as the
// layout's ownership rules require.  It is never used by the product library.
#include "../../orkan_b200/csrc/cuda/common.cuh"
#include "../../orkan_b200/csrc/cuda/dm_engine.cuh"
#include "../../orkan_b200/csrc/cuda/dm_phase.cuh"
#include "../../orkan_b200/csrc/cuda/pure.cuh"
#include "../../orkan_b200/csrc/cuda/pure_fused.cuh"
#include "../../orkan_b200/csrc/cuda/qaoa.cuh"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

using namespace orkan;

namespace {

struct EmuMem {
    double2* p;
    idx_t len;
    uint32_t* reads;
    uint32_t* writes;
    uint64_t* oob;
    double2 ld(idx_t i) const {
        if (i >= len) { ++*oob; return c2(0.0, 0.0); }
        ++reads[i];
        return p[i];
    }
    void st(idx_t i, double2 v) const {
        if (i >= len) { ++*oob; return; }
        ++writes[i];
        p[i] = v;
    }
    // asynchronous copy of the GPU path: lands immediately here; counted as one read per
    // element even when an element is copied to two shared-memory slots
    void cp(double2* dst, idx_t i) const {
        if (i >= len) { ++*oob; return; }
        if (i != last_cp) ++reads[i];
        last_cp = i;
        *dst = p[i];
    }
    mutable idx_t last_cp = ~idx_t(0);
    void cp16(double2* dst, idx_t i) const {
        if (i >= len) { ++*oob; return; }
        ++reads[i];
        *dst = p[i];
    }
    // asynchronous copy of a phase-table entry (not state storage): lands immediately here
    void cpg(double2* dst, const double2* src) const { *dst = *src; }
    // bulk copies of the GPU path (TMA): n consecutive elements, land immediately here
    void bulk_load(double2* sdst, idx_t i, unsigned n, void*) const {
        for (unsigned k = 0; k < n; ++k) sdst[k] = ld(i + k);
    }
    void bulk_store(idx_t i, const double2* ssrc, unsigned n) const {
        for (unsigned k = 0; k < n; ++k) st(i + k, ssrc[k]);
    }
};

struct EmuMemR {
    const double* p;
    idx_t len;
    uint64_t* oob;
    double ld(idx_t i) const {
        if (i >= len) { ++*oob; return 0.0; }
        return p[i];
    }
};

struct EmuMemC2 {
    const double2* p;
    idx_t len;
    uint64_t* oob;
    double2 ld(idx_t i) const {
        if (i >= len) { ++*oob; return c2(0.0, 0.0); }
        return p[i];
    }
};

// Cost vector accessor of the QAOA fill: the FP64 cost of amplitude i, or runs of byte
// costs (len counts the allocated bytes, whole 16-byte units).
template <class CostT>
struct EmuCost {
    const CostT* p;
    idx_t len;
    uint64_t* oob;
    void cpw(double* dst, idx_t i) const {
        if (i >= len) { ++*oob; return; }
        *dst = (double)p[i];
    }
    // byte costs: `bytes` costs from i (a multiple of bytes), within the allocated bytes
    void cpb(uint8_t* dst, idx_t i, unsigned bytes) const {
        if ((bytes != 4 && bytes != 8 && bytes != 16) || i % bytes || i + bytes > len) { ++*oob; return; }
        memcpy(dst, reinterpret_cast<const uint8_t*>(p) + i, bytes);
    }
};

constexpr unsigned kSms = 148;

unsigned grid_for(idx_t per_block, idx_t total, unsigned cap) {
    idx_t g = (total + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

double2 ldc(const double* p, unsigned i) { return c2(p[2 * i], p[2 * i + 1]); }

template <class Map, class Op>
void run_engine(const EmuMem& mem, const Map& map, const DmGeom& g, const Op& op) {
    const unsigned grid = grid_for(1, g.items, kSms * 32u);
    std::vector<double2> vb((size_t)g.V() * g.P());
    std::vector<DmPos> pd(kDmMaxPos + 1);
    Op o = op;
    dm_orient(o, !Map::kMirrors);           // the packed layout stages rho^T
    for (unsigned b = 0; b < grid; ++b) {
        for (idx_t w = b; w < g.items; w += grid) {
            for (int phase = 0; phase < kDmPhases; ++phase) {
                const unsigned nthr = (phase == 1 || phase == 5) ? kDmIssueThreads : kDmBlock;
                for (unsigned t = 0; t < nthr; ++t)
                    dm_engine_item_phase(phase, mem, map, g, o, w, pd.data(), vb.data(), t, nthr);
            }
        }
    }
}

template <class Op>
int engine_dispatch(int layout, unsigned log_tile, double* rho, idx_t len, unsigned n, const DmGeom& g,
                    const Op& op, uint32_t* reads, uint32_t* writes, uint64_t* oob) {
    EmuMem mem{reinterpret_cast<double2*>(rho), len, reads, writes, oob};
    if (layout == 1) run_engine(mem, PackedMap{idx_t(1) << n}, g, op);
    else run_engine(mem, TiledMap{idx_t(1) << n, log_tile}, g, op);
    return 0;
}

unsigned ls_max_for(int layout, unsigned log_tile) { return layout == 2 ? log_tile : 6u; }

// block-side cap of the engine (the GPU default 64, or ORKAN_DM_MAX_V)
unsigned emu_max_v() {
    unsigned x = 64;
    if (const char* e = getenv("ORKAN_DM_MAX_V")) {
        const unsigned y = (unsigned)atoi(e);
        if (y == 8 || y == 16 || y == 32 || y == 64) x = y;
    }
    return x;
}

template <class Factor>
void run_phase(int layout, unsigned log_tile, const EmuMem& mem, unsigned n, const Factor& fac) {
    const PhaseGeom g = phase_geometry(n, layout == 2 ? log_tile : 5u);
    const unsigned grid = grid_for(1, g.items, kSms * 32u);
    for (unsigned b = 0; b < grid; ++b)
        for (idx_t w = b; w < g.items; w += grid) {
            double2 srow[32], scol[32];
            for (unsigned t = 0; t < kPhaseThreads; ++t) dm_phase_stage(g, fac, w, srow, scol, t, kPhaseThreads);
            for (unsigned t = 0; t < kPhaseThreads; ++t) {
                if (layout == 1) dm_phase_item(mem, PackedMap{idx_t(1) << n}, g, fac, w, t, kPhaseThreads, srow, scol);
                else dm_phase_item(mem, TiledMap{idx_t(1) << n, log_tile}, g, fac, w, t, kPhaseThreads, srow, scol);
            }
        }
}


// One instance through the fused QAOA passes 0..upto (the GPU launch plan with a single
// instance): full pass when n <= C, else p + 1 low/high passes of 2^C-amplitude chunks.
template <class CostT>
int run_qaoa(unsigned n, const CostT* cost, unsigned p, const double* gamma, const double* beta, unsigned C,
             unsigned nthr, unsigned upto, double* psi, double* mean, uint32_t* reads, uint32_t* writes,
             uint64_t* oob) {
    const bool full = n <= C;
    if (p == 0 || nthr % 32 || (!full && 2 * C < n) || C > kQaoaMaxC) return -1;
    const idx_t dim = idx_t(1) << n;
    std::vector<QaoaRx> rx(p);
    std::vector<double2> table(1, c2(1.0, 0.0));
    unsigned tstride = 1;
    for (unsigned k = 0; k < p; ++k)
        rx[k] = qaoa_rx_coeffs(cos(2.0 * beta[k] / 2.0), sin(2.0 * beta[k] / 2.0), n, C);
    if (sizeof(CostT) == 1) {
        unsigned cmax = 0;
        for (idx_t x = 0; x < dim; ++x) cmax = cost[x] > cmax ? (unsigned)cost[x] : cmax;
        tstride = cmax + 1;
        table.assign((size_t)p * tstride, c2(0.0, 0.0));
        for (unsigned k = 0; k < p; ++k)
            for (unsigned c = 0; c <= cmax; ++c) {
                double sn, cs;
                sincos((double)c * gamma[k], &sn, &cs);
                table[(size_t)k * tstride + c] = c2(cs, sn);
            }
    }
    QaoaInst I;
    I.psi = reinterpret_cast<double2*>(psi);
    I.cost = cost;
    I.item0 = 0;
    I.n = n;
    I.pos = 0;
    const EmuMem mem{reinterpret_cast<double2*>(psi), dim, reads, writes, oob};
    const idx_t clen = sizeof(CostT) == 1 ? ((dim + 15) / 16) * 16 : dim;
    const EmuCost<CostT> cmem{cost, clen, oob};
    // byte costs of the high passes: the transposed array (qaoa_cost_t_index), as the batch
    // context builds it for the chunk size
    std::vector<CostT> cost_t;
    if (sizeof(CostT) == 1 && !full) {
        cost_t.assign((size_t)clen, CostT(0));
        for (idx_t x = 0; x < dim; ++x) cost_t[(size_t)qaoa_cost_t_index(n, C, x)] = cost[x];
    }
    const EmuCost<CostT> cmem_t{cost_t.empty() ? cost : cost_t.data(), clen, oob};
    const unsigned npass = full ? 1 : p + 1;
    for (unsigned j = 0; j < npass && j <= upto; ++j) {
        QaoaPass P;
        P.inst = &I;
        P.ninst = 1;
        P.kind = full ? kQaoaFull : ((j % 2 == 0) ? kQaoaLow : kQaoaHigh);
        P.C = full ? n : C;
        P.items = qaoa_items(n, P.C, P.kind);
        P.gamma = gamma;
        std::vector<double> partial(P.items, 0.0);
        P.partial = partial.data();
        P.p = p;
        P.pass = full ? 0 : j;
        qaoa_pass_setup(P, n);
        const QaoaTables T{table.data(), rx.data(), tstride};
        const QaoaPlan& pl = P.plan;
        std::vector<unsigned char> smem(qaoa_smem_bytes<CostT>(P.C, nthr, 1));
        const QaoaSmem<CostT> S = qaoa_smem_at<CostT>(smem.data(), P.C, nthr, 1, 0);
        const bool transposed = P.kind == kQaoaHigh && !cost_t.empty();
        I.cost = transposed ? static_cast<const void*>(cost_t.data()) : static_cast<const void*>(cost);
        const EmuCost<CostT>& cm = transposed ? cmem_t : cmem;
        for (idx_t w = 0; w < P.items; ++w) {
            for (unsigned t = 0; t < nthr; ++t) qaoa_fill<CostT>(P, T, I, pl, mem, cm, w, S, t, nthr);
            for (unsigned st = 0; st < qaoa_stages(pl); ++st)
                for (unsigned t = 0; t < nthr; ++t) qaoa_stage<CostT>(P, T, I, pl, mem, w, st, S, t, nthr);
        }
        if (pl.measure) {
            double s = 0.0;
            for (idx_t w = 0; w < P.items; ++w) s += partial[w];
            *mean = s;
        }
    }
    return 0;
}

}  // namespace

extern "C" {

// All entry points: data arrays are interleaved complex; reads/writes are per-element
// counters (zeroed by the caller); *oob receives the number of out-of-range accesses.
// Return 0, or -1 when the launch parameters are rejected (as the CUDA layer would).

int emu_dm_unitary(int layout, unsigned log_tile, double* rho, uint64_t len, unsigned n, unsigned k,
                   const unsigned* qubits, const double* u, uint32_t* reads, uint32_t* writes, uint64_t* oob) {
    DmGeom g;
    if (!dm_geometry(n, k, qubits, ls_max_for(layout, log_tile), &g, emu_max_v())) return -1;
    if (k == 1) {
        OpMix1 op;
        for (unsigned i = 0; i < 4; ++i) op.u[i] = ldc(u, i);
        return engine_dispatch(layout, log_tile, rho, len, n, g, op, reads, writes, oob);
    }
    OpMix2 op;
    for (unsigned i = 0; i < 16; ++i) op.u[i] = ldc(u, i);
    return engine_dispatch(layout, log_tile, rho, len, n, g, op, reads, writes, oob);
}

int emu_dm_monomial(int layout, unsigned log_tile, double* rho, uint64_t len, unsigned n, unsigned k,
                    const unsigned* qubits, const unsigned* src, const double* phase, uint32_t* reads,
                    uint32_t* writes, uint64_t* oob) {
    OpMonomial op;
    for (unsigned y = 0; y < 8; ++y) { op.src[y] = y; op.phase[y] = c2(1.0, 0.0); }
    for (unsigned y = 0; y < (1u << k); ++y) { op.src[y] = src[y]; op.phase[y] = ldc(phase, y); }
    DmGeom g;
    if (!dm_monomial_setup(n, k, qubits, op, ls_max_for(layout, log_tile), emu_max_v(), &g)) return -1;
    return engine_dispatch(layout, log_tile, rho, len, n, g, op, reads, writes, oob);
}

int emu_dm_superop1(int layout, unsigned log_tile, double* rho, uint64_t len, unsigned n, unsigned target,
                    const double* sop, uint32_t* reads, uint32_t* writes, uint64_t* oob) {
    OpSuper1 op;
    for (unsigned i = 0; i < 16; ++i) op.s[i] = ldc(sop, i);
    DmGeom g;
    const unsigned q[1] = {target};
    if (!dm_geometry(n, 1, q, ls_max_for(layout, log_tile), &g, emu_max_v())) return -1;
    return engine_dispatch(layout, log_tile, rho, len, n, g, op, reads, writes, oob);
}

int emu_dm_superop2(int layout, unsigned log_tile, double* rho, uint64_t len, unsigned n, unsigned q0, unsigned q1,
                    const double* sop, uint32_t* reads, uint32_t* writes, uint64_t* oob) {
    OpSuper2 op;
    for (unsigned i = 0; i < 256; ++i) op.s[i] = ldc(sop, i);
    DmGeom g;
    const unsigned q[2] = {q0, q1};
    if (!dm_geometry(n, 2, q, ls_max_for(layout, log_tile), &g, emu_max_v())) return -1;
    return engine_dispatch(layout, log_tile, rho, len, n, g, op, reads, writes, oob);
}

// Geometry of channel_2q on (q0, q1): -1 when there is none, else bit 0 set when the items
// take the tensor-core form and bit 1 when the staged block holds the 256 superoperator
// entries that the engine stages there before the first item (the device code stages only
// when both hold); out = {V, P, dynamic shared-memory bytes of an engine block}.
int emu_super2_geometry(int layout, unsigned log_tile, unsigned n, unsigned q0, unsigned q1, uint64_t* out) {
    DmGeom g;
    const unsigned q[2] = {q0, q1};
    if (!dm_geometry(n, 2, q, ls_max_for(layout, log_tile), &g, emu_max_v())) return -1;
    out[0] = g.V();
    out[1] = g.P();
    out[2] = dm_block_smem_bytes(g);
    return (super2_mma_form(g, kDmBlock) ? 1 : 0) | (super2_stage_fits(g) ? 2 : 0);
}

int emu_dm_phase(int layout, unsigned log_tile, double* rho, uint64_t len, unsigned n, unsigned k,
                 const unsigned* qubits, const double* phase, uint32_t* reads, uint32_t* writes, uint64_t* oob) {
    EmuMem mem{reinterpret_cast<double2*>(rho), len, reads, writes, oob};
    if (k == 1 && phase[0] == 1.0 && phase[1] == 0.0) {
        GateFactor1 f1;
        f1.q = qubits[0];
        f1.ph1 = ldc(phase, 1);
        run_phase(layout, log_tile, mem, n, f1);
        return 0;
    }
    {                                                   // controlled phase, as the GPU launcher picks it
        bool ctrl = true;
        for (unsigned y = 0; y + 1 < (1u << k); ++y) ctrl = ctrl && phase[2 * y] == 1.0 && phase[2 * y + 1] == 0.0;
        if (ctrl) {
            GateFactorCtrl fc;
            fc.mask = 0;
            for (unsigned j = 0; j < k; ++j) fc.mask |= 1ull << qubits[j];
            fc.ph = ldc(phase, (1u << k) - 1);
            run_phase(layout, log_tile, mem, n, fc);
            return 0;
        }
    }
    GateFactor fac;
    fac.k = k;
    for (unsigned j = 0; j < 3; ++j) fac.q[j] = j < k ? qubits[j] : 0;
    for (unsigned y = 0; y < 8; ++y) fac.phase[y] = y < (1u << k) ? ldc(phase, y) : c2(1.0, 0.0);
    run_phase(layout, log_tile, mem, n, fac);
    return 0;
}

// exp_diag on a density matrix: phase table from diag, then the phase pass (as the GPU path).
int emu_dm_exp_diag(int layout, unsigned log_tile, double* rho, uint64_t len, unsigned n, const double* diag,
                    double t, uint32_t* reads, uint32_t* writes, uint64_t* oob) {
    if (t == 0.0) return 0;
    const idx_t d = idx_t(1) << n;
    std::vector<double2> tab(d);
    for (idx_t x = 0; x < d; ++x) {
        double sn, cs;
        sincos(diag[x] * t, &sn, &cs);
        tab[x] = c2(cs, sn);
    }
    TableFactor<EmuMemC2> fac{EmuMemC2{tab.data(), d, oob}};
    EmuMem mem{reinterpret_cast<double2*>(rho), len, reads, writes, oob};
    run_phase(layout, log_tile, mem, n, fac);
    return 0;
}

int emu_pure_gate1(double* psi, unsigned n, unsigned target, int op, double c, double s, uint32_t* reads,
                   uint32_t* writes, uint64_t* oob) {
    if (n < 1 || target >= n) return -1;
    const idx_t npairs = idx_t(1) << (n - 1);
    const unsigned grid = grid_for(kPureThreads * kVec, npairs, kSms * 8u);
    const idx_t nthr = (idx_t)grid * kPureThreads;
    EmuMem mem{reinterpret_cast<double2*>(psi), idx_t(1) << n, reads, writes, oob};
    for (idx_t tid = 0; tid < nthr; ++tid) {
        switch (op) {
#define ORKAN_EMU_CASE(OPC) case OPC: pure1q_thread<OPC>(mem, npairs, target, c, s, tid, nthr); break;
            ORKAN_EMU_CASE(kOpX) ORKAN_EMU_CASE(kOpY) ORKAN_EMU_CASE(kOpZ) ORKAN_EMU_CASE(kOpH)
            ORKAN_EMU_CASE(kOpS) ORKAN_EMU_CASE(kOpSdg) ORKAN_EMU_CASE(kOpT) ORKAN_EMU_CASE(kOpTdg)
            ORKAN_EMU_CASE(kOpHy) ORKAN_EMU_CASE(kOpRx) ORKAN_EMU_CASE(kOpRy) ORKAN_EMU_CASE(kOpRz)
            ORKAN_EMU_CASE(kOpP)
#undef ORKAN_EMU_CASE
            default: return -1;
        }
    }
    return 0;
}

int emu_pure_gate2(double* psi, unsigned n, unsigned qa, unsigned qb, int op, uint32_t* reads, uint32_t* writes,
                   uint64_t* oob) {
    if (n < 2 || qa >= n || qb >= n || qa == qb) return -1;
    const idx_t nq = idx_t(1) << (n - 2);
    const unsigned grid = grid_for(kPureThreads * kVec, nq, kSms * 8u);
    const idx_t nthr = (idx_t)grid * kPureThreads;
    EmuMem mem{reinterpret_cast<double2*>(psi), idx_t(1) << n, reads, writes, oob};
    for (idx_t tid = 0; tid < nthr; ++tid) {
        switch (op) {
            case kOpCX: pure2q_thread<kOpCX>(mem, nq, qa, qb, tid, nthr); break;
            case kOpCY: pure2q_thread<kOpCY>(mem, nq, qa, qb, tid, nthr); break;
            case kOpCZ: pure2q_thread<kOpCZ>(mem, nq, qa, qb, tid, nthr); break;
            case kOpSwap: pure2q_thread<kOpSwap>(mem, nq, qa, qb, tid, nthr); break;
            default: return -1;
        }
    }
    return 0;
}

int emu_pure_ccx(double* psi, unsigned n, unsigned c1, unsigned c2q, unsigned t, uint32_t* reads, uint32_t* writes,
                 uint64_t* oob) {
    if (n < 3) return -1;
    const idx_t no = idx_t(1) << (n - 3);
    const unsigned grid = grid_for(kPureThreads * kVec, no, kSms * 8u);
    const idx_t nthr = (idx_t)grid * kPureThreads;
    EmuMem mem{reinterpret_cast<double2*>(psi), idx_t(1) << n, reads, writes, oob};
    for (idx_t tid = 0; tid < nthr; ++tid) pure_ccx_thread(mem, no, c1, c2q, t, tid, nthr);
    return 0;
}

int emu_pure_exp_diag(double* psi, unsigned n, const double* diag, double t, uint32_t* reads, uint32_t* writes,
                      uint64_t* oob) {
    const idx_t d = idx_t(1) << n;
    const unsigned grid = grid_for(kPureThreads * kVec, d, kSms * 8u);
    const idx_t nthr = (idx_t)grid * kPureThreads;
    EmuMem mem{reinterpret_cast<double2*>(psi), d, reads, writes, oob};
    EmuMemR dg{diag, d, oob};
    for (idx_t tid = 0; tid < nthr; ++tid) pure_exp_diag_thread(mem, dg, d, t, tid, nthr);
    return 0;
}

int emu_fill(double* data, uint64_t len, double re, double im, unsigned corner_log_tile, uint64_t corner_dim,
             uint32_t* reads, uint32_t* writes, uint64_t* oob) {
    const unsigned grid = grid_for(kPureThreads * 4, len, kSms * 8u);
    const idx_t nthr = (idx_t)grid * kPureThreads;
    EmuMem mem{reinterpret_cast<double2*>(data), len, reads, writes, oob};
    for (idx_t tid = 0; tid < nthr; ++tid) fill_thread(mem, len, c2(re, im), corner_log_tile, corner_dim, tid, nthr);
    return 0;
}

// A fused run of statevector gates (k_pure_fused): every block of the grid, phase by phase
// (offset table; per chunk: load, each register stage, store), with a block-local chunk buffer.
int emu_pure_fused(double* psi, unsigned n, unsigned log_chunk, unsigned ngates, const orkan_fgate_t* gates,
                   unsigned grid_cap, uint32_t* reads, uint32_t* writes, uint64_t* oob) {
    FusedPlan P;
    if (!fused_plan(n, log_chunk, ngates, gates, &P)) return -1;
    const unsigned nthr = kFuseThreads;
    const idx_t nch = P.nchunks();
    const unsigned grid = grid_for(1, nch, grid_cap ? grid_cap : kSms * 4u);
    EmuMem mem{reinterpret_cast<double2*>(psi), idx_t(1) << n, reads, writes, oob};
    std::vector<double2> buf(P.chunk());
    std::vector<idx_t> tab(P.ntab());
    for (unsigned b = 0; b < grid; ++b) {
        for (unsigned t = 0; t < nthr; ++t) fused_table(P, tab.data(), t, nthr);
        for (idx_t ch = b; ch < nch; ch += grid) {
            const idx_t base = fused_base(P, ch);
            for (unsigned t = 0; t < nthr; ++t) fused_load(mem, P, tab.data(), base, buf.data(), t, nthr);
            for (unsigned st = 0; st < P.nstages; ++st)
                for (unsigned t = 0; t < nthr; ++t) fused_stage(P, st, base, buf.data(), t, nthr);
            for (unsigned t = 0; t < nthr; ++t) fused_store(mem, P, tab.data(), base, buf.data(), t, nthr);
        }
    }
    return 0;
}

unsigned long long emu_fused_need(const orkan_fgate_t* g) { return fused_need(*g); }

// Register stages the plan cuts a run into (-1: the run does not fit).
int emu_fused_stages(unsigned n, unsigned log_chunk, unsigned ngates, const orkan_fgate_t* gates) {
    FusedPlan P;
    if (!fused_plan(n, log_chunk, ngates, gates, &P)) return -1;
    return (int)P.nstages;
}

// Shared-memory layout of the QAOA pass kernel: 1 when every region is aligned for all
// chunk sizes 0..13 and ring depths 1, 2, for both cost types.
int emu_qaoa_smem_aligned(void) {
    for (unsigned C = 0; C <= kQaoaMaxC; ++C)
        for (unsigned ring = 1; ring <= 2; ++ring)
            if (!qaoa_smem_aligned<uint8_t>(C, ring) || !qaoa_smem_aligned<double>(C, ring)) return 0;
    return 1;
}

// Fused QAOA passes of one instance; byte_cost selects byte costs (cost_b) over doubles.
int emu_qaoa(unsigned n, const double* cost_d, const uint8_t* cost_b, int byte_cost, unsigned p, const double* gamma,
             const double* beta, unsigned C, unsigned nthr, unsigned upto, double* psi, double* mean,
             uint32_t* reads, uint32_t* writes, uint64_t* oob) {
    if (byte_cost) return run_qaoa<uint8_t>(n, cost_b, p, gamma, beta, C, nthr, upto, psi, mean, reads, writes, oob);
    return run_qaoa<double>(n, cost_d, p, gamma, beta, C, nthr, upto, psi, mean, reads, writes, oob);
}

}  // extern "C"
