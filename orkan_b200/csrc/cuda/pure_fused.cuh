// pure_fused.cuh - several consecutive statevector gates in one pass over HBM.
//
// The reference applies every gate as its own pass over the 2^n amplitudes
// (src/gate/gate_pure.c:33-48, TRAVERSE_PURE_1Q, and the quarter/eighth loops of
// gate_pure.c:282-434).  Here a run of gates is applied chunk by chunk: a chunk is the set of
// 2^C amplitudes whose indices differ only in C chosen "local" qubits, it is loaded into
// shared memory once, every gate of the run is applied to it there, and it is stored once.
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

enum FKind : unsigned char {
    kFMix = 0,    // pair_op<op> on (bit t clear, bit t set) where the local controls are set
    kFPhase,      // the |1>-half of a diagonal 1-qubit op on local bit t (local controls)
    kFRz,         // Rz on local bit t (both halves change)
    kFSwap,       // exchange of the (t=1, a=0) and (t=0, a=1) amplitudes
    kFScale       // diagonal op on non-local bits: every amplitude of the chunk changes
};

struct FGate {
    unsigned char kind, op, t, a;
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
    FGate g[kFuseMaxGates];
    ORKAN_HD unsigned chunk() const { return 1u << C; }
    ORKAN_HD idx_t nchunks() const { return idx_t(1) << (n - C); }
    ORKAN_HD unsigned ntab() const { return 1u << (C - m); }
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
    return true;
}

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
            if (j < N) buf[j] = v[u];
        }
    }
}

template <class Mem>
ORKAN_HD void fused_store(const Mem& mem, const FusedPlan& P, const idx_t* tab, idx_t base, const double2* buf,
                          unsigned tid, unsigned nthr) {
    const unsigned N = P.chunk();
    for (unsigned j = tid; j < N; j += nthr) mem.st(base + fused_off(P, tab, j), buf[j]);
}

// Does gate g act on the chunk at base?  (Its non-local controls are all set.)
ORKAN_HD bool fused_active(const FGate& g, idx_t base) { return (base & g.gmask) == g.gmask; }

template <int OP>
ORKAN_HD void fused_mix(const FGate& g, double2* buf, unsigned half, unsigned tid, unsigned nthr) {
    const unsigned bt = 1u << g.t;
    for (unsigned p = tid; p < half; p += nthr) {
        const unsigned i0 = (unsigned)insert0(p, g.t);
        if ((i0 & g.lmask) != g.lmask) continue;
        double2 a = buf[i0], b = buf[i0 | bt];
        pair_op<OP>(a, b, g.c, g.s);
        buf[i0] = a;
        buf[i0 | bt] = b;
    }
}

template <int OP>
ORKAN_HD void fused_phase(const FGate& g, double2* buf, unsigned half, unsigned tid, unsigned nthr) {
    const unsigned bt = 1u << g.t;
    for (unsigned p = tid; p < half; p += nthr) {
        const unsigned i1 = (unsigned)insert0(p, g.t) | bt;
        if ((i1 & g.lmask) != g.lmask) continue;
        double2 a = c2(0.0, 0.0), b = buf[i1];
        pair_op<OP>(a, b, g.c, g.s);
        buf[i1] = b;
    }
}

template <int OP>
ORKAN_HD void fused_scale(const FGate& g, double2* buf, unsigned N, unsigned tid, unsigned nthr) {
    for (unsigned j = tid; j < N; j += nthr) {
        double2 a = c2(0.0, 0.0), b = buf[j];
        pair_op<OP>(a, b, g.c, g.s);
        buf[j] = b;
    }
}

// Rz on a non-local bit: every amplitude takes the |0> factor (bit clear) or the |1> factor.
ORKAN_HD void fused_scale_rz(const FGate& g, double2* buf, unsigned N, bool one, unsigned tid, unsigned nthr) {
    for (unsigned j = tid; j < N; j += nthr) {
        double2 a = buf[j], b = buf[j];
        pair_op<kOpRz>(a, b, g.c, g.s);
        buf[j] = one ? b : a;
    }
}

// One gate on the staged chunk (all threads of the block; a barrier follows).
ORKAN_HD void fused_gate(const FusedPlan& P, const FGate& g, idx_t base, double2* buf, unsigned tid, unsigned nthr) {
    const unsigned N = P.chunk(), half = N >> 1;
    switch (g.kind) {
        case kFMix:
            switch (g.op) {
                case kOpX: fused_mix<kOpX>(g, buf, half, tid, nthr); break;
                case kOpY: fused_mix<kOpY>(g, buf, half, tid, nthr); break;
                case kOpH: fused_mix<kOpH>(g, buf, half, tid, nthr); break;
                case kOpHy: fused_mix<kOpHy>(g, buf, half, tid, nthr); break;
                case kOpRx: fused_mix<kOpRx>(g, buf, half, tid, nthr); break;
                default: fused_mix<kOpRy>(g, buf, half, tid, nthr); break;
            }
            break;
        case kFPhase:
            switch (g.op) {
                case kOpZ: fused_phase<kOpZ>(g, buf, half, tid, nthr); break;
                case kOpS: fused_phase<kOpS>(g, buf, half, tid, nthr); break;
                case kOpSdg: fused_phase<kOpSdg>(g, buf, half, tid, nthr); break;
                case kOpT: fused_phase<kOpT>(g, buf, half, tid, nthr); break;
                case kOpTdg: fused_phase<kOpTdg>(g, buf, half, tid, nthr); break;
                default: fused_phase<kOpP>(g, buf, half, tid, nthr); break;
            }
            break;
        case kFRz:
            fused_mix<kOpRz>(g, buf, half, tid, nthr);
            break;
        case kFSwap: {
            const unsigned lo = g.t < g.a ? g.t : g.a, hi = g.t < g.a ? g.a : g.t;
            const unsigned bt = 1u << g.t, ba = 1u << g.a;
            for (unsigned p = tid; p < (N >> 2); p += nthr) {
                const unsigned i00 = (unsigned)insert0(insert0(p, lo), hi);
                const double2 x = buf[i00 | bt], y = buf[i00 | ba];
                buf[i00 | bt] = y;
                buf[i00 | ba] = x;
            }
            break;
        }
        default:   // kFScale
            if (g.op == kOpRz) {
                fused_scale_rz(g, buf, N, (base & g.gbit) != 0, tid, nthr);
            } else {
                switch (g.op) {
                    case kOpZ: fused_scale<kOpZ>(g, buf, N, tid, nthr); break;
                    case kOpS: fused_scale<kOpS>(g, buf, N, tid, nthr); break;
                    case kOpSdg: fused_scale<kOpSdg>(g, buf, N, tid, nthr); break;
                    case kOpT: fused_scale<kOpT>(g, buf, N, tid, nthr); break;
                    case kOpTdg: fused_scale<kOpTdg>(g, buf, N, tid, nthr); break;
                    default: fused_scale<kOpP>(g, buf, N, tid, nthr); break;
                }
            }
            break;
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
        for (unsigned gi = 0; gi < P.ngates; ++gi) {
            const FGate& g = P.g[gi];
            if (!fused_active(g, base)) continue;        // the same for every thread of the block
            fused_gate(P, g, base, fbuf, tid, nthr);
            __syncthreads();
        }
        fused_store(mem, P, tab, base, fbuf, tid, nthr);
        __syncthreads();
    }
}
#endif

}  // namespace orkan
