// pure_fused.cuh - several consecutive statevector gates in one pass over HBM.
//
// The reference applies every gate as its own pass over the 2^n amplitudes
// (src/gate/gate_pure.c:33-48, TRAVERSE_PURE_1Q, and the quarter/eighth loops of
// gate_pure.c:282-434).  Here a run of gates is applied chunk by chunk: a chunk is the set of
// 2^C amplitudes whose indices differ only in C chosen "local" qubits, it is loaded into
// shared memory once, every gate of the run is applied to it there, and it is stored once.
// Inside the chunk the run is cut into stages: a stage holds consecutive gates whose mixed
// qubits fit a group of 4 local qubits; every thread takes the 16 amplitudes of a set that
// differ only in the group's qubits into registers, applies all of the stage's gates there,
// and puts them back, so the shared memory is read and written once per stage, not per gate.
//
// * A gate can join a run when the qubits it mixes are local: the target of X, Y, H, Hy, Rx,
//   Ry, CX, CY and CCX, both qubits of SWAP.  Controls and diagonal gates (Z, S, Sdg, T, Tdg,
//   P, Rz, CZ) may sit on any qubit: a non-local bit is constant over a chunk, so a non-local
//   control becomes a condition on the chunk and a non-local diagonal gate a factor applied
//   to the whole chunk (or to nothing).
// * The local set always holds the lowest qubits that are free, at least qubits 0-2, so a
//   chunk is made of contiguous runs of >= 8 amplitudes (128-byte lines): loads and stores
//   stay coalesced wherever the mixed qubits lie.
// * Every gate uses the same per-pair arithmetic as its one-gate kernel (pair_op of
//   pure.cuh), so a fused run gives bit-identical results to the gates applied one by one.
//
// The index logic is written as per-thread, per-phase __host__ __device__ functions so the
// CPU emulator of the test suite runs it with bounds-checked memory before any GPU run.
#pragma once

#include "common.cuh"
#include "pure.cuh"

#include "../../../include/orkan_cu.h"

namespace orkan {

constexpr unsigned kFuseMaxGates = 48;   // gates of one fused launch
constexpr unsigned kFuseMaxLog = 12;     // chunk of at most 2^12 amplitudes (64 KB)
constexpr unsigned kFuseThreads = 256;
constexpr unsigned kFuseVec = 8;         // loads a thread issues before it stores any
constexpr unsigned kFuseGroup = 3;       // local qubits of a register stage (8 amplitudes)

enum FKind : unsigned char {
    kFMix = 0,    // pair_op<op> on (bit t clear, bit t set) where the local controls are set
    kFPhase,      // the |1>-half of a diagonal 1-qubit op on local bit t (local controls)
    kFRz,         // Rz on local bit t (both halves change)
    kFSwap,       // exchange of the (t=1, a=0) and (t=0, a=1) amplitudes
    kFScale       // diagonal op on non-local bits: every amplitude of the chunk changes
};

struct FGate {
    unsigned char kind, op, t, a;
    unsigned char rt, ra;      // kFMix / kFSwap: positions of t and a in the stage's group
    unsigned char pad_[2];
    unsigned lmask;            // local control bits (chunk index)
    unsigned long long gmask;  // the gate acts on a chunk only when all these global bits are set
    unsigned long long gbit;   // kFScale Rz: the global bit that picks the |0> or |1> factor
    double c, s;
};

struct FusedPlan {
    unsigned n, C, m;          // qubits, log2 chunk, length of the run of local bits 0..m-1
    unsigned ngates;
    unsigned long long nlmask; // global bits that are not local (the chunk id's bits)
    unsigned char lq[kFuseMaxLog];   // global position of local bit i (ascending)
    unsigned K;                // qubits of a stage's group: min(kFuseGroup, C)
    unsigned nstages;
    unsigned char st_first[kFuseMaxGates + 1];     // first gate of stage s; st_first[nstages] = ngates
    unsigned char st_g[kFuseMaxGates][kFuseGroup]; // local bits of stage s's group, ascending
    FGate g[kFuseMaxGates];
    ORKAN_HD unsigned chunk() const { return 1u << C; }
    ORKAN_HD idx_t nchunks() const { return idx_t(1) << (n - C); }
    ORKAN_HD unsigned ntab() const { return 1u << (C - m); }
    ORKAN_HD unsigned sets() const { return 1u << (C - K); }
};

// Global qubits a gate mixes (must be local) as a bit mask; ~0 for an unknown op.
inline unsigned long long fused_need(const orkan_fgate_t& q) {
    switch (q.op) {
        case ORKAN_OP_X: case ORKAN_OP_Y: case ORKAN_OP_H: case ORKAN_OP_HY: case ORKAN_OP_RX: case ORKAN_OP_RY:
            return 1ull << q.q[0];
        case ORKAN_OP_Z: case ORKAN_OP_S: case ORKAN_OP_SDG: case ORKAN_OP_T: case ORKAN_OP_TDG: case ORKAN_OP_P:
        case ORKAN_OP_RZ: case ORKAN_FOP_CZ:
            return 0;
        case ORKAN_FOP_CX: case ORKAN_FOP_CY: return 1ull << q.q[1];
        case ORKAN_FOP_SWAP: return (1ull << q.q[0]) | (1ull << q.q[1]);
        case ORKAN_FOP_CCX: return 1ull << q.q[2];
        default: return ~0ull;
    }
}

inline unsigned fused_arity(int op) {
    return op < ORKAN_FOP_CX ? 1u : (op == ORKAN_FOP_CCX ? 3u : 2u);
}

// Build the plan of a run on an n-qubit statevector with chunks of 2^C amplitudes.  False
// when the run does not fit (too many mixed qubits, bad qubits or op codes, too many gates).
inline bool fused_plan(unsigned n, unsigned C, unsigned ngates, const orkan_fgate_t* gates, FusedPlan* P) {
    if (n < 1 || n > 62 || C < 1 || C > kFuseMaxLog || C > n || ngates < 1 || ngates > kFuseMaxGates) return false;
    const unsigned long long all = (n >= 64) ? ~0ull : ((1ull << n) - 1ull);
    unsigned long long need = 7ull & all;
    for (unsigned i = 0; i < ngates; ++i) {
        const orkan_fgate_t& q = gates[i];
        const unsigned k = fused_arity(q.op);
        if (q.op < 0 || (q.op > ORKAN_OP_P && q.op < ORKAN_FOP_CX) || q.op > ORKAN_FOP_CCX) return false;
        for (unsigned j = 0; j < k; ++j) {
            if (q.q[j] >= n) return false;
            for (unsigned l = 0; l < j; ++l) if (q.q[l] == q.q[j]) return false;
        }
        need |= fused_need(q);
    }
    if (popc64(need) > C) return false;
    for (unsigned b = 0; b < n && popc64(need) < C; ++b) need |= 1ull << b;   // lowest free bits
    P->n = n;
    P->C = C;
    P->ngates = ngates;
    P->nlmask = all & ~need;
    unsigned pos[64];
    unsigned i = 0;
    for (unsigned b = 0; b < n; ++b)
        if ((need >> b) & 1ull) { P->lq[i] = (unsigned char)b; pos[b] = i++; }
    P->m = 0;
    while (P->m < C && P->lq[P->m] == P->m) ++P->m;
    for (unsigned gi = 0; gi < ngates; ++gi) {
        const orkan_fgate_t& q = gates[gi];
        FGate& f = P->g[gi];
        f.kind = kFMix;
        f.op = 0;
        f.t = f.a = 0;
        f.lmask = 0;
        f.gmask = f.gbit = 0;
        f.c = q.c;
        f.s = q.s;
        auto local = [&](unsigned b) { return ((need >> b) & 1ull) != 0; };
        auto control = [&](unsigned b) {
            if (local(b)) f.lmask |= 1u << pos[b];
            else f.gmask |= 1ull << b;
        };
        switch (q.op) {
            case ORKAN_OP_X: case ORKAN_OP_Y: case ORKAN_OP_H: case ORKAN_OP_HY: case ORKAN_OP_RX: case ORKAN_OP_RY:
                f.kind = kFMix; f.op = (unsigned char)q.op; f.t = (unsigned char)pos[q.q[0]];
                break;
            case ORKAN_OP_Z: case ORKAN_OP_S: case ORKAN_OP_SDG: case ORKAN_OP_T: case ORKAN_OP_TDG: case ORKAN_OP_P:
                f.op = (unsigned char)q.op;
                if (local(q.q[0])) { f.kind = kFPhase; f.t = (unsigned char)pos[q.q[0]]; }
                else { f.kind = kFScale; f.gmask = 1ull << q.q[0]; }
                break;
            case ORKAN_OP_RZ:
                f.op = (unsigned char)q.op;
                if (local(q.q[0])) { f.kind = kFRz; f.t = (unsigned char)pos[q.q[0]]; }
                else { f.kind = kFScale; f.gbit = 1ull << q.q[0]; }
                break;
            case ORKAN_FOP_CX: case ORKAN_FOP_CY:
                f.kind = kFMix; f.op = q.op == ORKAN_FOP_CX ? (unsigned char)kOpX : (unsigned char)kOpY;
                f.t = (unsigned char)pos[q.q[1]];
                control(q.q[0]);
                break;
            case ORKAN_FOP_CZ:
                f.op = (unsigned char)kOpZ;
                if (local(q.q[1])) { f.kind = kFPhase; f.t = (unsigned char)pos[q.q[1]]; control(q.q[0]); }
                else if (local(q.q[0])) { f.kind = kFPhase; f.t = (unsigned char)pos[q.q[0]]; control(q.q[1]); }
                else { f.kind = kFScale; f.gmask = (1ull << q.q[0]) | (1ull << q.q[1]); }
                break;
            case ORKAN_FOP_SWAP:
                f.kind = kFSwap; f.t = (unsigned char)pos[q.q[0]]; f.a = (unsigned char)pos[q.q[1]];
                break;
            case ORKAN_FOP_CCX:
                f.kind = kFMix; f.op = (unsigned char)kOpX; f.t = (unsigned char)pos[q.q[2]];
                control(q.q[0]);
                control(q.q[1]);
                break;
            default: return false;
        }
    }
    // stages: consecutive gates whose mixed local bits fit a group of K bits; a group with
    // fewer is filled with the lowest other local bits
    P->K = C < kFuseGroup ? C : kFuseGroup;
    P->nstages = 0;
    unsigned cur = 0;
    auto close = [&](unsigned first, unsigned last) {
        for (unsigned b = 0; b < C && popc64(cur) < P->K; ++b) cur |= 1u << b;
        unsigned char* gb = P->st_g[P->nstages];
        unsigned k = 0;
        for (unsigned b = 0; b < C; ++b)
            if ((cur >> b) & 1u) gb[k++] = (unsigned char)b;
        for (; k < kFuseGroup; ++k) gb[k] = 0;
        for (unsigned gi = first; gi < last; ++gi) {
            FGate& f = P->g[gi];
            f.rt = f.ra = 0;
            for (unsigned r = 0; r < P->K; ++r) {
                if (gb[r] == f.t) f.rt = (unsigned char)r;
                if (gb[r] == f.a) f.ra = (unsigned char)r;
            }
        }
        P->st_first[P->nstages++] = (unsigned char)first;
        cur = 0;
    };
    unsigned first = 0;
    for (unsigned gi = 0; gi < ngates; ++gi) {
        const FGate& f = P->g[gi];
        const unsigned need = f.kind == kFMix ? (1u << f.t) : f.kind == kFSwap ? ((1u << f.t) | (1u << f.a)) : 0u;
        if (popc64(cur | need) > P->K) {
            close(first, gi);
            first = gi;
        }
        cur |= need;
    }
    close(first, ngates);
    P->st_first[P->nstages] = (unsigned char)ngates;
    return true;
}

// Shared-memory slot of chunk index s: the low 3 bits XORed with the three 3-bit fields above
// them, so the 8 lanes of a quarter warp that differ in bits of distinct residues mod 3 (and
// any 8 consecutive indices) hit distinct 16-byte bank groups.
ORKAN_HD unsigned fused_phys(unsigned s) { return s ^ (((s >> 3) ^ (s >> 6) ^ (s >> 9)) & 7u); }

// Global index of the chunk's amplitude 0: the chunk id's bits deposited on the non-local bits.
ORKAN_HD idx_t fused_base(const FusedPlan& P, idx_t chunk) {
    idx_t base = 0;
    unsigned long long rest = P.nlmask;
    while (rest && chunk) {
        const unsigned b = ctz64(rest);
        base |= (chunk & 1u) << b;
        chunk >>= 1;
        rest &= rest - 1ull;
    }
    return base;
}

// Offset table of the local bits above the contiguous run: tab[h] = sum of bit i of h at
// global position lq[m + i].
ORKAN_HD void fused_table(const FusedPlan& P, idx_t* tab, unsigned tid, unsigned nthr) {
    for (unsigned h = tid; h < P.ntab(); h += nthr) {
        idx_t o = 0;
        for (unsigned i = 0; i + P.m < P.C; ++i) o |= idx_t((h >> i) & 1u) << P.lq[P.m + i];
        tab[h] = o;
    }
}

ORKAN_HD idx_t fused_off(const FusedPlan& P, const idx_t* tab, unsigned j) {
    return tab[j >> P.m] + (j & ((1u << P.m) - 1u));
}

template <class Mem>
ORKAN_HD void fused_load(const Mem& mem, const FusedPlan& P, const idx_t* tab, idx_t base, double2* buf,
                         unsigned tid, unsigned nthr) {
    const unsigned N = P.chunk();
    for (unsigned j0 = tid; j0 < N; j0 += kFuseVec * nthr) {
        double2 v[kFuseVec];
#pragma unroll
        for (unsigned u = 0; u < kFuseVec; ++u) {
            const unsigned j = j0 + u * nthr;
            if (j < N) v[u] = mem.ld(base + fused_off(P, tab, j));
        }
#pragma unroll
        for (unsigned u = 0; u < kFuseVec; ++u) {
            const unsigned j = j0 + u * nthr;
            if (j < N) buf[fused_phys(j)] = v[u];
        }
    }
}

template <class Mem>
ORKAN_HD void fused_store(const Mem& mem, const FusedPlan& P, const idx_t* tab, idx_t base, const double2* buf,
                          unsigned tid, unsigned nthr) {
    const unsigned N = P.chunk();
    for (unsigned j = tid; j < N; j += nthr) mem.st(base + fused_off(P, tab, j), buf[fused_phys(j)]);
}

// Does gate g act on the chunk at base?  (Its non-local controls are all set.)
ORKAN_HD bool fused_active(const FGate& g, idx_t base) { return (base & g.gmask) == g.gmask; }

// ---- register stages -------------------------------------------------------------------
// v[j] holds the amplitude at chunk index idx[j] = set base | (bit b of j at group bit g[b]).

template <int OP, int RT, int NV>
ORKAN_HD void reg_mix(double2 (&v)[NV], const unsigned (&idx)[NV], const FGate& g) {
    const double c = g.c, s = g.s;
    if (g.lmask == 0) {                              // no local control: every pair
#pragma unroll
        for (int j = 0; j < NV; ++j)
            if (!(j & (1 << RT))) pair_op<OP>(v[j], v[j | (1 << RT)], c, s);
        return;
    }
#pragma unroll
    for (int j = 0; j < NV; ++j)
        if (!(j & (1 << RT)) && (idx[j] & g.lmask) == g.lmask) pair_op<OP>(v[j], v[j | (1 << RT)], c, s);
}

template <int OP, int NV>
ORKAN_HD void reg_mix_at(double2 (&v)[NV], const unsigned (&idx)[NV], const FGate& g) {
    switch (g.rt) {
        case 0: reg_mix<OP, 0>(v, idx, g); break;
        case 1: if (NV > 2) reg_mix<OP, (NV > 2 ? 1 : 0)>(v, idx, g); break;
        case 2: if (NV > 4) reg_mix<OP, (NV > 4 ? 2 : 0)>(v, idx, g); break;
        default: if (NV > 8) reg_mix<OP, (NV > 8 ? 3 : 0)>(v, idx, g); break;
    }
}

// The |1>-half op of a diagonal gate on local bit t (its bit need not be in the group).
template <int OP, int NV>
ORKAN_HD void reg_phase(double2 (&v)[NV], const unsigned (&idx)[NV], const FGate& g) {
    const unsigned need = g.lmask | (1u << g.t);
#pragma unroll
    for (int j = 0; j < NV; ++j)
        if ((idx[j] & need) == need) {
            double2 a = c2(0.0, 0.0);
            pair_op<OP>(a, v[j], g.c, g.s);
        }
}

// Rz on local bit t: each amplitude takes the |0> or the |1> factor by its bit t (or, on a
// non-local bit, by the chunk's bit: `one`).
// The |1> factor is the |0> factor with s negated: (c x + s y, c y - s x) -> (c x - s y, c y + s x),
// the same roundings as pair_op<kOpRz>.
template <int NV>
ORKAN_HD void reg_rz(double2 (&v)[NV], const unsigned (&idx)[NV], const FGate& g, bool local, bool one) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const double s = (local ? ((idx[j] >> g.t) & 1u) != 0 : one) ? -g.s : g.s;
        v[j] = c2(lin2(g.c, v[j].x, s, v[j].y), lin2(g.c, v[j].y, -s, v[j].x));
    }
}

// A diagonal 1-qubit op's |1> factor on every amplitude (a non-local gate whose bits are set).
template <int OP, int NV>
ORKAN_HD void reg_scale(double2 (&v)[NV], const FGate& g) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        double2 a = c2(0.0, 0.0);
        pair_op<OP>(a, v[j], g.c, g.s);
    }
}

template <int RT, int RA, int NV>
ORKAN_HD void reg_swap(double2 (&v)[NV]) {
#pragma unroll
    for (int j = 0; j < NV; ++j)
        if (!(j & (1 << RT)) && !(j & (1 << RA))) {
            const double2 x = v[j | (1 << RT)];
            v[j | (1 << RT)] = v[j | (1 << RA)];
            v[j | (1 << RA)] = x;
        }
}

template <int NV>
ORKAN_HD void reg_swap_at(double2 (&v)[NV], unsigned rt, unsigned ra) {
    constexpr int K = NV >= 16 ? 4 : NV >= 8 ? 3 : NV >= 4 ? 2 : 1;
    const unsigned lo = rt < ra ? rt : ra, hi = rt < ra ? ra : rt;
    if (K < 2) return;
    switch (lo * 4 + hi) {
        case 1: reg_swap<0, 1>(v); break;
        case 2: if (K > 2) reg_swap<0, (K > 2 ? 2 : 1)>(v); break;
        case 3: if (K > 3) reg_swap<0, (K > 3 ? 3 : 1)>(v); break;
        case 6: if (K > 2) reg_swap<1, (K > 2 ? 2 : 0)>(v); break;
        case 7: if (K > 3) reg_swap<1, (K > 3 ? 3 : 0)>(v); break;
        default: if (K > 3) reg_swap<2, (K > 3 ? 3 : 0)>(v); break;   // (2, 3)
    }
}

// One gate of a stage on a thread's registers.
template <int NV>
ORKAN_HD void fused_apply(const FGate& g, double2 (&v)[NV], const unsigned (&idx)[NV], idx_t base) {
    switch (g.kind) {
        case kFMix:
            switch (g.op) {
                case kOpX: reg_mix_at<kOpX>(v, idx, g); break;
                case kOpY: reg_mix_at<kOpY>(v, idx, g); break;
                case kOpH: reg_mix_at<kOpH>(v, idx, g); break;
                case kOpHy: reg_mix_at<kOpHy>(v, idx, g); break;
                case kOpRx: reg_mix_at<kOpRx>(v, idx, g); break;
                default: reg_mix_at<kOpRy>(v, idx, g); break;
            }
            break;
        case kFPhase:
            switch (g.op) {
                case kOpZ: reg_phase<kOpZ>(v, idx, g); break;
                case kOpS: reg_phase<kOpS>(v, idx, g); break;
                case kOpSdg: reg_phase<kOpSdg>(v, idx, g); break;
                case kOpT: reg_phase<kOpT>(v, idx, g); break;
                case kOpTdg: reg_phase<kOpTdg>(v, idx, g); break;
                default: reg_phase<kOpP>(v, idx, g); break;
            }
            break;
        case kFRz:
            reg_rz(v, idx, g, true, false);
            break;
        case kFSwap:
            reg_swap_at(v, g.rt, g.ra);
            break;
        default:   // kFScale
            if (g.op == kOpRz) {
                reg_rz(v, idx, g, false, (base & g.gbit) != 0);
            } else {
                switch (g.op) {
                    case kOpZ: reg_scale<kOpZ>(v, g); break;
                    case kOpS: reg_scale<kOpS>(v, g); break;
                    case kOpSdg: reg_scale<kOpSdg>(v, g); break;
                    case kOpT: reg_scale<kOpT>(v, g); break;
                    case kOpTdg: reg_scale<kOpTdg>(v, g); break;
                    default: reg_scale<kOpP>(v, g); break;
                }
            }
            break;
    }
}

// Stage s of the run on the staged chunk (all threads of the block; a barrier follows).
// Thread tid takes sets tid, tid + nthr, ...: the set's 2^K amplitudes go to registers, every
// gate of the stage whose chunk condition holds is applied, and they go back.
template <int NV>
ORKAN_HD void fused_stage_k(const FusedPlan& P, unsigned s, idx_t base, double2* buf, unsigned tid, unsigned nthr) {
    constexpr int K = NV >= 16 ? 4 : NV >= 8 ? 3 : NV >= 4 ? 2 : 1;
    // element j of a set sits at set base | off[j]; the swizzle is linear over disjoint bits,
    // so its slot is phys(set base) ^ phys(off[j]), with phys(off[j]) formed once per stage
    unsigned off[NV], poff[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        unsigned o = 0;
#pragma unroll
        for (int b = 0; b < K; ++b)
            if ((j >> b) & 1) o |= 1u << P.st_g[s][b];
        off[j] = o;
        poff[j] = fused_phys(o);
    }
    const unsigned g0 = P.st_first[s], g1 = P.st_first[s + 1];
    for (unsigned r = tid; r < P.sets(); r += nthr) {
        unsigned sb = r;
        for (int b = 0; b < K; ++b) sb = (unsigned)insert0(sb, P.st_g[s][b]);   // ascending positions
        const unsigned psb = fused_phys(sb);
        double2 v[NV];
        unsigned idx[NV];
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            idx[j] = sb | off[j];
            v[j] = buf[psb ^ poff[j]];
        }
        for (unsigned gi = g0; gi < g1; ++gi) {
            const FGate& g = P.g[gi];
            if (fused_active(g, base)) fused_apply(g, v, idx, base);
        }
#pragma unroll
        for (int j = 0; j < NV; ++j) buf[psb ^ poff[j]] = v[j];
    }
}

ORKAN_HD void fused_stage(const FusedPlan& P, unsigned s, idx_t base, double2* buf, unsigned tid, unsigned nthr) {
    switch (P.K) {
        case 4: fused_stage_k<(kFuseGroup >= 4 ? 16 : 8)>(P, s, base, buf, tid, nthr); break;
        case 3: fused_stage_k<8>(P, s, base, buf, tid, nthr); break;
        case 2: fused_stage_k<4>(P, s, base, buf, tid, nthr); break;
        default: fused_stage_k<2>(P, s, base, buf, tid, nthr); break;
    }
}

// Shared memory of one block: the chunk and the offset table.
ORKAN_HD size_t fused_smem_bytes(const FusedPlan& P) {
    return (size_t)P.chunk() * sizeof(double2) + (size_t)P.ntab() * sizeof(idx_t);
}

#ifdef __CUDACC__
// Persistent blocks walk the chunks; every gate whose chunk condition holds is applied in
// shared memory between one load and one store of the chunk.
__global__ void __launch_bounds__(kFuseThreads) k_pure_fused(DevMem mem, const __grid_constant__ FusedPlan P) {
    extern __shared__ __align__(16) double2 fbuf[];
    idx_t* tab = reinterpret_cast<idx_t*>(fbuf + P.chunk());
    const unsigned tid = threadIdx.x, nthr = blockDim.x;
    fused_table(P, tab, tid, nthr);
    __syncthreads();
    const idx_t nch = P.nchunks();
    for (idx_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        const idx_t base = fused_base(P, ch);
        fused_load(mem, P, tab, base, fbuf, tid, nthr);
        __syncthreads();
        for (unsigned st = 0; st < P.nstages; ++st) {
            fused_stage(P, st, base, fbuf, tid, nthr);
            __syncthreads();
        }
        fused_store(mem, P, tab, base, fbuf, tid, nthr);
        __syncthreads();
    }
}
#endif

}  // namespace orkan
