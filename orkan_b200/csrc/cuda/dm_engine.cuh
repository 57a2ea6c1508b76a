// dm_engine.cuh - rho -> U rho U^dagger (and 1-qubit superoperators) on the packed and
// tiled density-matrix layouts, as one fused row-and-column update per block of the
// matrix staged in shared memory.
//
// Reference behaviour followed: the 2x2-block update of src/gate/packed/gate_packed_1q.c:65-104
// (conjugate read/write of elements that fall in the upper triangle), the three tiled
// sub-cases of src/gate/tiled/gate_tiled_h.c:28-223 (all-lower quads, mirrored T(tc1,tr0)
// access, diagonal tile pair with mirror writes) and the superoperator block update of
// src/channel/channel_packed.c:48-120 / channel_tiled.c:52-185.
//
// Design.  A gate acts on k <= 3 qubits.  The matrix is cut into S x S sub-tiles
// (S = 2^ls).  Gate qubits below ls act inside a sub-tile; the h gate qubits at or
// above ls pair up sub-tiles.  One work item ("super-tile") is the set of rows
// R_a = (rowbase | offset(a)) * S + [0,S) and columns C_b likewise, a,b in [0, 2^h):
// it is closed under the gate's action on rows and on columns.  The item is staged in
// shared memory as a dense V x V block (V = S * 2^h) of the full Hermitian matrix:
// sub-tiles stored in the lower triangle are copied, sub-tiles of the upper triangle
// are filled with the conjugate transpose of their stored partner, and diagonal
// sub-tiles are completed from their lower half.  Threads then apply the gate to
// disjoint element groups of the block (no cross-thread hazards), and the stored
// sub-tiles are written back, regenerating the upper half of every diagonal tile of
// the tiled layout from its lower half, so the tiled mirror invariant holds exactly.
//
// Ownership: item (u, v), u >= v, owns every stored sub-tile whose segment indices,
// with the high gate bits cleared, are (u, v) or (v, u); each stored element is read
// once and written once per launch (the CPU emulator in tests/emu checks this).
#pragma once

#include "common.cuh"
#include <math.h>

namespace orkan {

constexpr unsigned kDmThreads = 256;
constexpr unsigned kDmMaxV = 64;            // largest virtual block side
constexpr unsigned kDmMaxElems = kDmMaxV * kDmMaxV;

// Geometry of one launch (computed on the host by dm_geometry()).
struct DmGeom {
    idx_t d;            // 2^n
    unsigned n;
    unsigned ls;        // log2 of the sub-tile side S
    unsigned h;         // gate qubits with position >= ls
    unsigned hb[3];     // their positions in segment-index space (q - ls), ascending
    unsigned k;         // gate qubits
    unsigned vbit[3];   // virtual-index bit of gate qubit j; j = 0 is the MSB of the local index
    idx_t nbase;        // base segments per dimension: (d >> ls) >> h
    idx_t items;        // nbase * (nbase + 1) / 2
    unsigned fixmask;   // bit l set: local index l is left in place with phase 1 by the gate
                        // (monomial gates only; an element whose row and column are both
                        // fixed is unchanged and is neither loaded nor stored)
    unsigned long long fixrows;  // the same as a mask over virtual indices (dm_fixed_rows)
    ORKAN_HD unsigned S() const { return 1u << ls; }
    ORKAN_HD unsigned V() const { return 1u << (ls + h); }
    ORKAN_HD unsigned P() const { return V() + 1; }    // smem row pitch (padded)
};

// Choose the sub-tile side: the largest S (<= smax) with V^2 <= kDmMaxElems.
// qubits[j] is gate qubit j, qubits[0] the most significant bit of the local index.
inline bool dm_geometry(unsigned n, unsigned k, const unsigned* qubits, unsigned ls_max, DmGeom* g) {
    if (k < 1 || k > 3 || n < k) return false;
    for (unsigned j = 0; j < k; ++j) {
        if (qubits[j] >= n) return false;
        for (unsigned i = 0; i < j; ++i) if (qubits[i] == qubits[j]) return false;
    }
    unsigned ls = ls_max < n ? ls_max : n;
    for (;; --ls) {
        unsigned h = 0;
        for (unsigned j = 0; j < k; ++j) h += (qubits[j] >= ls);
        if ((1ull << (2 * (ls + h))) <= kDmMaxElems || ls == 0) {
            g->d = idx_t(1) << n;
            g->n = n;
            g->ls = ls;
            g->h = h;
            g->k = k;
            // high qubits in ascending order -> hb, and their virtual bits ls + rank
            unsigned hq[3], nh = 0;
            for (unsigned j = 0; j < k; ++j) if (qubits[j] >= ls) hq[nh++] = qubits[j];
            for (unsigned a = 0; a < nh; ++a)
                for (unsigned b = a + 1; b < nh; ++b)
                    if (hq[b] < hq[a]) { unsigned t = hq[a]; hq[a] = hq[b]; hq[b] = t; }
            for (unsigned a = 0; a < 3; ++a) g->hb[a] = a < nh ? hq[a] - ls : 0;
            for (unsigned j = 0; j < k; ++j) {
                if (qubits[j] < ls) {
                    g->vbit[j] = qubits[j];
                } else {
                    unsigned rank = 0;
                    while (hq[rank] != qubits[j]) ++rank;
                    g->vbit[j] = ls + rank;
                }
            }
            for (unsigned j = k; j < 3; ++j) g->vbit[j] = 0;
            g->nbase = (g->d >> ls) >> h;
            g->items = g->nbase * (g->nbase + 1) / 2;
            g->fixmask = 0;
            g->fixrows = 0;
            return true;
        }
        if (ls == 0) return false;
    }
}

// Sub-tile classes of position (a, b) of an item.
enum : int { kSubDirect = 0, kSubDiag = 1, kSubTransposed = 2, kSubSkip = 3 };

// Per-position descriptor of an item, built once per item in shared memory so that each
// element's storage index, shared-memory slot(s) and skip test cost a few integer ops.
// A "line" is a run of S consecutive storage elements of a stored sub-tile (a column
// segment of the packed layout, a row segment of a tile); p is the offset along it.
struct DmPos {
    idx_t gbase;   // storage index of element (line 0, p 0) of the stored sub-tile
    idx_t mbase;   // tiled: storage index of the mirror of (line 0, p 0); written at mbase + p*T + line
    idx_t gcol;    // packed: d - PC - 1, the column-start increment per line
    int d0, dl, dp;  // direct shared-memory slot: d0 + line*dl + p*dp
    int c0, cl, cp;  // conjugated shared-memory slot
    int fconst;      // virtual index constant along a line is fconst + line
    int fvar;        // virtual index varying along a line is fvar + p
    int cls;         // kSub*
    int has_c;       // a direct sub-tile that also fills its transposed position (diagonal item)
    int mirror;      // tiled: the stored sub-tile lies in a diagonal tile; rewrite its mirror
    int pad_;
};
constexpr unsigned kDmMaxPos = 64;                     // 4^h with h <= 3
constexpr unsigned kDmPosBytes = kDmMaxPos * sizeof(DmPos);

// Shared memory of one block: descriptors, then the V x (V + 1) staged block.
ORKAN_HD size_t dm_smem_bytes(const DmGeom& g) { return kDmPosBytes + (size_t)g.V() * g.P() * 16; }

// Virtual-index bit masks of fixed rows/columns (monomial gates): bit x set when local(x)
// is left in place with phase 1.  V <= 64, so one 64-bit word.
ORKAN_HD unsigned dm_get_local(unsigned x, const unsigned* vbit, unsigned k);
inline unsigned long long dm_fixed_rows(const DmGeom& g) {
    if (!g.fixmask) return 0ull;
    unsigned long long m = 0;
    for (unsigned x = 0; x < g.V(); ++x)
        if ((g.fixmask >> dm_get_local(x, g.vbit, g.k)) & 1u) m |= 1ull << x;
    return m;
}

// Build the descriptors of item w (threads tid < 4^h, one position each).
template <class Map>
ORKAN_HD void dm_setup(const Map& map, const DmGeom& g, idx_t w, DmPos* pd, unsigned tid, unsigned nthr) {
    const unsigned h = g.h, ls = g.ls, S = g.S(), P = g.P();
    const unsigned npos = 1u << (2 * h);
    if (tid >= npos) return;
    idx_t u, v;
    tri_unrank(w, &u, &v);
    const bool diag_item = (u == v);
    const idx_t rb = insert0_sorted(u, g.hb, h), cb = insert0_sorted(v, g.hb, h);
    for (unsigned t = tid; t < npos; t += nthr) {
        const unsigned a = t >> h, b = t & ((1u << h) - 1);
        const idx_t R = (rb | spread_bits(a, g.hb, h)) << ls;
        const idx_t C = (cb | spread_bits(b, g.hb, h)) << ls;
        DmPos q;
        q.mbase = 0;
        q.gcol = 0;
        q.has_c = 0;
        q.mirror = 0;
        q.pad_ = 0;
        q.d0 = q.dl = q.dp = q.c0 = q.cl = q.cp = 0;
        q.fconst = q.fvar = 0;
        const int aS = (int)(a * S), bS = (int)(b * S);
        if (R > C) {
            q.cls = kSubDirect;
            q.gbase = map.at(R, C);
            q.has_c = diag_item ? 1 : 0;
            if (Map::kRowContig) {       // packed: line = column j, p = row i
                q.d0 = aS * (int)P + bS; q.dl = 1; q.dp = (int)P;
                q.c0 = bS * (int)P + aS; q.cl = (int)P; q.cp = 1;
                q.fconst = bS; q.fvar = aS;
                q.gcol = map.d - C - 1;
            } else {                     // tiled: line = row i, p = column j
                q.d0 = aS * (int)P + bS; q.dl = (int)P; q.dp = 1;
                q.c0 = bS * (int)P + aS; q.cl = 1; q.cp = (int)P;
                q.fconst = aS; q.fvar = bS;
                if (map.same_storage_block(R, C)) { q.mirror = 1; q.mbase = map.at(C, R); }
            }
        } else if (R == C) {
            q.cls = kSubDiag;
            q.gbase = map.at(R, R);
            q.d0 = aS * (int)P + aS;
            q.c0 = aS * (int)P + aS;
            q.fconst = aS; q.fvar = aS;
            if (Map::kRowContig) { q.dl = 1; q.dp = (int)P; q.cl = (int)P; q.cp = 1; q.gcol = map.d - R - 1; }
            else                 { q.dl = (int)P; q.dp = 1; q.cl = 1; q.cp = (int)P; }
        } else if (!diag_item) {
            q.cls = kSubTransposed;
            q.gbase = map.at(C, R);      // stored partner (C, R)
            if (Map::kRowContig) {       // stored (C + p, R + line) is virtual (aS + line, bS + p), conjugated
                q.c0 = aS * (int)P + bS; q.cl = (int)P; q.cp = 1;
                q.fconst = aS; q.fvar = bS;
                q.gcol = map.d - R - 1;
            } else {                     // stored (C + line, R + p) is virtual (aS + p, bS + line), conjugated
                q.c0 = aS * (int)P + bS; q.cl = 1; q.cp = (int)P;
                q.fconst = bS; q.fvar = aS;
                if (map.same_storage_block(C, R)) { q.mirror = 1; q.mbase = map.at(R, C); }
            }
        } else {
            q.cls = kSubSkip;
            q.gbase = 0;
        }
        pd[t] = q;
    }
}

// Storage index of element (line, p) of a position's stored sub-tile.
template <class Map>
ORKAN_HD idx_t dm_addr(const Map& map, const DmPos& q, unsigned line, unsigned p) {
    if (Map::kRowContig) return q.gbase + (idx_t)line * q.gcol - (idx_t)((line * (line - 1)) >> 1) + p;
    return q.gbase + ((idx_t)line << map.log_tdim()) + p;
}

ORKAN_HD bool dm_skip(unsigned long long fm, const DmPos& q, unsigned line, unsigned p) {
    return fm && ((fm >> (q.fconst + line)) & (fm >> (q.fvar + p)) & 1ull);
}

// Load rules: which of the element's slots the load fills (bit 0 direct, bit 1 conjugate).
template <class Map>
ORKAN_HD unsigned dm_load_slots(const DmPos& q, unsigned line, unsigned p) {
    switch (q.cls) {
        case kSubDirect: return 1u | (q.has_c ? 2u : 0u);
        case kSubTransposed: return 2u;
        case kSubDiag:
            if (Map::kRowContig) return p >= line ? (1u | (p > line ? 2u : 0u)) : 0u;
            return p <= line ? (1u | (p < line ? 2u : 0u)) : 0u;
        default: return 0u;
    }
}

// Stage one item into the shared block vb (pitch P) with asynchronous 16-byte global->shared
// copies (cp.async): no register staging, so a block keeps a whole item in flight while it
// computes and stores the previous one.  An element that must also appear conjugated
// (upper half of a diagonal sub-tile, the transposed copy of a sub-tile of a diagonal
// item, every element of a transposed sub-tile) is copied raw into its conjugate slot and
// fixed up by the same thread after its copies have landed (dm_fixup).
template <class Map, class Mem>
ORKAN_HD void dm_issue(const Mem& mem, const Map& map, const DmGeom& g, const DmPos* pd, double2* vb,
                       unsigned tid, unsigned nthr) {
    const unsigned ls = g.ls, S = g.S();
    const unsigned total = 1u << (2 * (ls + g.h));
    const unsigned long long fm = g.fixrows;
    for (unsigned f = tid; f < total; f += nthr) {
        const DmPos& q = pd[f >> (2 * ls)];
        const unsigned e = f & ((1u << (2 * ls)) - 1), line = e >> ls, p = e & (S - 1);
        const unsigned which = dm_load_slots<Map>(q, line, p);
        if (!which || dm_skip(fm, q, line, p)) continue;
        const idx_t a = dm_addr(map, q, line, p);
        if (which & 1u) mem.cp(vb + (q.d0 + (int)line * q.dl + (int)p * q.dp), a);
        if (which & 2u) mem.cp(vb + (q.c0 + (int)line * q.cl + (int)p * q.cp), a);
    }
}

// Conjugate the slots this thread filled through its conjugate copies (after they landed).
template <class Map>
ORKAN_HD void dm_fixup(const DmGeom& g, const DmPos* pd, double2* vb, unsigned tid, unsigned nthr) {
    const unsigned ls = g.ls, S = g.S();
    const unsigned total = 1u << (2 * (ls + g.h));
    const unsigned long long fm = g.fixrows;
    for (unsigned f = tid; f < total; f += nthr) {
        const DmPos& q = pd[f >> (2 * ls)];
        const unsigned e = f & ((1u << (2 * ls)) - 1), line = e >> ls, p = e & (S - 1);
        if (!(dm_load_slots<Map>(q, line, p) & 2u) || dm_skip(fm, q, line, p)) continue;
        double2& x = vb[q.c0 + (int)line * q.cl + (int)p * q.cp];
        x.y = -x.y;
    }
}

// Write one item back, regenerating tiled mirrors and the upper half of diagonal tiles.
template <class Map, class Mem>
ORKAN_HD void dm_store(const Mem& mem, const Map& map, const DmGeom& g, const DmPos* pd, const double2* vb,
                       unsigned tid, unsigned nthr) {
    const unsigned ls = g.ls, S = g.S();
    const unsigned total = 1u << (2 * (ls + g.h));
    const unsigned long long fm = g.fixrows;
    for (unsigned f = tid; f < total; f += nthr) {
        const DmPos& q = pd[f >> (2 * ls)];
        if (q.cls == kSubSkip) continue;
        const unsigned e = f & ((1u << (2 * ls)) - 1), line = e >> ls, p = e & (S - 1);
        if (dm_skip(fm, q, line, p)) continue;
        double2 val;
        if (q.cls == kSubDirect) {
            val = vb[q.d0 + (int)line * q.dl + (int)p * q.dp];
        } else if (q.cls == kSubTransposed) {
            val = cconj(vb[q.c0 + (int)line * q.cl + (int)p * q.cp]);
        } else if (Map::kRowContig) {                   // packed diagonal sub-tile: lower half only
            if (p < line) continue;
            val = vb[q.d0 + (int)line * q.dl + (int)p * q.dp];
        } else {                                        // tiled diagonal sub-tile: both halves
            val = p <= line ? vb[q.d0 + (int)line * q.dl + (int)p * q.dp]
                            : cconj(vb[q.c0 + (int)line * q.cl + (int)p * q.cp]);
        }
        mem.st(dm_addr(map, q, line, p), val);
        if (Map::kMirrors && q.mirror)
            mem.st(q.mbase + ((idx_t)p << map.log_tdim()) + line, cconj(val));
    }
}

// ---------------------------------------------------------------------------------
// Group operations on the staged block.  Each thread owns whole groups, so compute
// needs no synchronisation between threads.
// ---------------------------------------------------------------------------------

// Virtual index with the local-index bits of gate qubits j placed (j = 0 is the MSB).
ORKAN_HD unsigned dm_set_local(unsigned x, unsigned loc, const unsigned* vbit, unsigned k) {
    for (unsigned j = 0; j < k; ++j) {
        const unsigned bit = (loc >> (k - 1 - j)) & 1u;
        x = (x & ~(1u << vbit[j])) | (bit << vbit[j]);
    }
    return x;
}
ORKAN_HD unsigned dm_get_local(unsigned x, const unsigned* vbit, unsigned k) {
    unsigned loc = 0;
    for (unsigned j = 0; j < k; ++j) loc = (loc << 1) | ((x >> vbit[j]) & 1u);
    return loc;
}

// Dense 1-qubit unitary U (row-major u[2*r + c]):  G' = U G U^dagger on 2x2 groups.
struct OpMix1 {
    double2 u[4];
    ORKAN_HD void operator()(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr) const {
        const unsigned V = g.V(), P = g.P(), half = V >> 1, vbq = g.vbit[0];
        const unsigned groups = half * half;
        for (unsigned t = tid; t < groups; t += nthr) {
            const unsigned r0 = (unsigned)insert0(t / half, vbq), c0 = (unsigned)insert0(t % half, vbq);
            const unsigned r1 = r0 | (1u << vbq), c1 = c0 | (1u << vbq);
            const double2 x00 = vb[r0 * P + c0], x01 = vb[r0 * P + c1];
            const double2 x10 = vb[r1 * P + c0], x11 = vb[r1 * P + c1];
            // rows: Y = U X
            const double2 y00 = cadd(cmul(u[0], x00), cmul(u[1], x10));
            const double2 y01 = cadd(cmul(u[0], x01), cmul(u[1], x11));
            const double2 y10 = cadd(cmul(u[2], x00), cmul(u[3], x10));
            const double2 y11 = cadd(cmul(u[2], x01), cmul(u[3], x11));
            // columns: Z = Y U^dagger, Z[i][j] = sum_m Y[i][m] conj(U[j][m])
            vb[r0 * P + c0] = cadd(cmulc(y00, u[0]), cmulc(y01, u[1]));
            vb[r0 * P + c1] = cadd(cmulc(y00, u[2]), cmulc(y01, u[3]));
            vb[r1 * P + c0] = cadd(cmulc(y10, u[0]), cmulc(y11, u[1]));
            vb[r1 * P + c1] = cadd(cmulc(y10, u[2]), cmulc(y11, u[3]));
        }
    }
};

// Dense 2-qubit unitary U (row-major u[4*r + c], local index = 2*bit(q0) + bit(q1)).
struct OpMix2 {
    double2 u[16];
    ORKAN_HD void operator()(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr) const {
        const unsigned V = g.V(), P = g.P(), quarter = V >> 2;
        unsigned asc[2] = {g.vbit[0] < g.vbit[1] ? g.vbit[0] : g.vbit[1],
                           g.vbit[0] < g.vbit[1] ? g.vbit[1] : g.vbit[0]};
        const unsigned groups = quarter * quarter;
        for (unsigned t = tid; t < groups; t += nthr) {
            const unsigned rb = (unsigned)insert0_sorted(t / quarter, asc, 2);
            const unsigned cb = (unsigned)insert0_sorted(t % quarter, asc, 2);
            unsigned ri[4], ci[4];
            for (unsigned l = 0; l < 4; ++l) {
                ri[l] = dm_set_local(rb, l, g.vbit, 2);
                ci[l] = dm_set_local(cb, l, g.vbit, 2);
            }
            double2 y[4][4];
            for (unsigned r = 0; r < 4; ++r)
                for (unsigned c = 0; c < 4; ++c) {
                    double2 acc = c2(0.0, 0.0);
                    for (unsigned m = 0; m < 4; ++m) acc = cadd(acc, cmul(u[4 * r + m], vb[ri[m] * P + ci[c]]));
                    y[r][c] = acc;
                }
            for (unsigned r = 0; r < 4; ++r)
                for (unsigned c = 0; c < 4; ++c) {
                    double2 acc = c2(0.0, 0.0);
                    for (unsigned m = 0; m < 4; ++m) acc = cadd(acc, cmulc(y[r][m], u[4 * c + m]));
                    vb[ri[r] * P + ci[c]] = acc;
                }
        }
    }
};

// 1-qubit superoperator (row-major s[4*m + j]) on vec = (x00, x01, x10, x11).
struct OpSuper1 {
    double2 s[16];
    ORKAN_HD void operator()(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr) const {
        const unsigned V = g.V(), P = g.P(), half = V >> 1, vbq = g.vbit[0];
        const unsigned groups = half * half;
        for (unsigned t = tid; t < groups; t += nthr) {
            const unsigned r0 = (unsigned)insert0(t / half, vbq), c0 = (unsigned)insert0(t % half, vbq);
            const unsigned r1 = r0 | (1u << vbq), c1 = c0 | (1u << vbq);
            const unsigned idx[4] = {r0 * P + c0, r0 * P + c1, r1 * P + c0, r1 * P + c1};
            double2 x[4];
            for (unsigned m = 0; m < 4; ++m) x[m] = vb[idx[m]];
            for (unsigned m = 0; m < 4; ++m) {
                double2 acc = c2(0.0, 0.0);
                for (unsigned j = 0; j < 4; ++j) acc = cadd(acc, cmul(s[4 * m + j], x[j]));
                vb[idx[m]] = acc;
            }
        }
    }
};

// Monomial gate U|x> with an involutive permutation (X, Y, CX, CY, SWAP, CCX ...):
// (U psi)[y] = phase[y] * psi[src[y]] on the local index, src[src[y]] == y.
// Element pairs (y, z) <-> (src y, src z) are 2-cycles; the thread owning the
// smaller flat index of a pair updates both.
struct OpMonomial {
    unsigned src[8];
    double2 phase[8];
    ORKAN_HD void operator()(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr) const {
        const unsigned V = g.V(), P = g.P(), k = g.k;
        const unsigned total = V * V;
        for (unsigned f = tid; f < total; f += nthr) {
            const unsigned r = f / V, c = f % V;
            const unsigned lr = dm_get_local(r, g.vbit, k), lc = dm_get_local(c, g.vbit, k);
            const unsigned r2 = dm_set_local(r, src[lr], g.vbit, k), c2i = dm_set_local(c, src[lc], g.vbit, k);
            const unsigned f2 = r2 * V + c2i;
            if (f2 < f) continue;
            const double2 fa = cmulc(phase[lr], phase[lc]);
            if (f2 == f) {
                vb[r * P + c] = cmul(fa, vb[r * P + c]);
            } else {
                const double2 fb = cmulc(phase[src[lr]], phase[src[lc]]);
                const double2 va = vb[r * P + c], vb2 = vb[r2 * P + c2i];
                vb[r * P + c] = cmul(fa, vb2);
                vb[r2 * P + c2i] = cmul(fb, va);
            }
        }
    }
};

// Local indices the monomial gate leaves in place with phase exactly 1.
inline unsigned monomial_fixmask(const OpMonomial& op, unsigned m) {
    unsigned mask = 0;
    for (unsigned l = 0; l < m; ++l)
        if (op.src[l] == l && op.phase[l].x == 1.0 && op.phase[l].y == 0.0) mask |= 1u << l;
    return mask;
}

// One work item, phase by phase (the CPU emulator runs each phase for all threads
// before the next; the kernel below overlaps items with a two-stage pipeline).
template <class Map, class Mem, class Op>
ORKAN_HD void dm_engine_item_phase(int phase, const Mem& mem, const Map& map, const DmGeom& g, const Op& op,
                                   idx_t w, DmPos* pd, double2* vb, unsigned tid, unsigned nthr) {
    if (phase == 0) dm_setup(map, g, w, pd, tid, nthr);
    else if (phase == 1) dm_issue(mem, map, g, pd, vb, tid, nthr);
    else if (phase == 2) dm_fixup<Map>(g, pd, vb, tid, nthr);
    else if (phase == 3) op(g, vb, tid, nthr);
    else dm_store(mem, map, g, pd, vb, tid, nthr);
}

constexpr unsigned kDmBlock = 512;          // threads of the pipelined engine block

// Shared memory of one pipelined block: two descriptor sets and two staged blocks.
ORKAN_HD size_t dm_pipe_smem_bytes(const DmGeom& g) { return 2 * dm_smem_bytes(g); }

#ifdef __CUDACC__
struct DevMemAsync : DevMem {
    __device__ __forceinline__ void cp(double2* sdst, idx_t i) const {
        const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(p + i) : "memory");
    }
};
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Persistent, double-buffered engine: block b handles items b, b + G, b + 2G, ...; the
// copies of the next item are in flight while the current one is computed and stored.
template <class Map, class Op>
__global__ void __launch_bounds__(kDmBlock) k_dm_engine(DevMemAsync mem, Map map, DmGeom g, Op op) {
    extern __shared__ double2 smem[];
    const size_t half = dm_smem_bytes(g) / sizeof(double2);
    DmPos* pd[2] = {reinterpret_cast<DmPos*>(smem), reinterpret_cast<DmPos*>(smem + half)};
    double2* vb[2] = {smem + kDmPosBytes / sizeof(double2), smem + half + kDmPosBytes / sizeof(double2)};
    const unsigned tid = threadIdx.x, nthr = blockDim.x;
    idx_t w = blockIdx.x;
    if (w >= g.items) return;
    dm_setup(map, g, w, pd[0], tid, nthr);
    __syncthreads();
    dm_issue(mem, map, g, pd[0], vb[0], tid, nthr);
    cp_commit();
    for (unsigned it = 0;; ++it) {
        const unsigned cur = it & 1u, nxt = cur ^ 1u;
        const idx_t wn = w + gridDim.x;
        if (wn < g.items) dm_setup(map, g, wn, pd[nxt], tid, nthr);
        __syncthreads();                                  // pd[nxt] ready; vb[nxt] free
        if (wn < g.items) dm_issue(mem, map, g, pd[nxt], vb[nxt], tid, nthr);
        cp_commit();
        cp_wait<1>();                                     // this thread's copies of item w landed
        dm_fixup<Map>(g, pd[cur], vb[cur], tid, nthr);
        __syncthreads();
        op(g, vb[cur], tid, nthr);
        __syncthreads();
        dm_store(mem, map, g, pd[cur], vb[cur], tid, nthr);
        if (wn >= g.items) break;
        w = wn;
        __syncthreads();                                  // vb[cur], pd[cur] free for item w + 2G
    }
    cp_wait<0>();
}
#endif

}  // namespace orkan
